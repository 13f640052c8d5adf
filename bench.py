#!/usr/bin/env python
"""Benchmark of the quantum-wire SBE step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c4|c1|c2|c3] [--chunk S]

Default workload: configuration 4, the serving stream (Poisson 2000
requests/s for 60 s; Nk in {64, 128, 256, 512, 1024} with p = {.3, .3, .2,
.15, .05}; 1-4 ps at dt = 1 fs; pulse area, detuning, FWHM and T2 as
configuration 1).  The line reports:

  value     the batched split form (exchange sums as exact int8-digit
            products on the tensor cores) on the stream's request mix as a
            resident batch (the first 16384 requests of the stream, about a
            saturated server's slots, inputs in HBM): a bench step advances
            every resident solve by S time steps (one CUDA-graph replay of
            one launch per size class); wire*k*steps/s = sum Nk * S / time.
  plain     the plain FP64 form of the same batch, same timing rules, and
            split_over_plain.
  accuracy  per-solve error of the split form against the plain FP64 form
            (which matches the FP64 oracle to <= 1e-10) over 4000 steps on
            the first 4096 solves: P(t), final p, n_e, n_h.
  e2e       the serving API (pulsesuite_b200.serve.Server.run): requests in
            from the host, continuous batching on the device, P(t) records
            and final states copied back to host memory; the saturated
            capacity of the split form on a backlog of the stream.
  serving   saturated capacity of both forms on the same backlog, and p50 /
            p99 solve latency of the Poisson stream served in real time (the
            split form on the whole 60 s; the plain form on a shorter slice).
  cpu_baseline            the CPU oracle (an OpenMP C restatement of the
                          reference's path) on a sample of the same mix, all
                          host cores;
  cpu_baseline_reference  the reference's own Numba path (imported from
                          baseline/_ref), full-matrix RHS + rk4_dpc, timed
                          per Nk and weighted by the mix (large Nk
                          extrapolated).

Timing: W untimed bench steps, then K bench steps each bracketed by CUDA
events on the launching stream, with a 256 MiB write between them (L2 is
126 MB) outside the events; barrier + synchronize around the whole loop;
max over ranks.  `--impl reference` times the CPU oracle on the host cores
on the same workload and prints the same line shape.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

L2_FLUSH_BYTES = 256 << 20
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the step
# kernels, from one ncu capture of a 20-step call on the configuration-4
# request mix (16384 solves; profiles/split_rk4_kernel_c4_mix.md,
# profiles/sbe_f64_kernel_c4_mix.md):
#   split, state resident in shared memory: per element and launch (the
#     FP64 state read once and written once)
#   split, state in the workspace (groups whose grid does not fit shared
#     memory): per element and time step (the FP32 stage state streams
#     through L2 and, beyond its capacity, DRAM every stage)
#   plain: per element and launch
DRAM_SPLIT_RES_PER_ELEMENT = 75.0e6 / 1.770048e6
DRAM_SPLIT_WS_PER_ELEMENT_STEP = 2.043e9 / (2.116608e6 * 20)
DRAM_PLAIN_PER_ELEMENT = (72.03e6 + 43.39e6) / (1.770048e6 + 1.267712e6)
TRAFFIC_SOURCE = ("ncu dram bytes per element (resident state, per launch) and per element "
                  "and step (workspace state) of a 20-step capture on the c4 mix, applied to "
                  "this step's launches")
METRIC = "SBE wire*k*steps/s at <=1e-6 rel err vs FP64 (batched vs plain); p50/p99 latency"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c4", choices=["c1", "c2", "c3", "c4", "pstd"])
    ap.add_argument("--chunk", type=int, default=100, help="time steps per bench step")
    ap.add_argument("--form", default="split", choices=["plain", "split"],
                    help="split int8-digit tensor-core kernel or plain FP64 kernel")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain-form comparison of the split run")
    ap.add_argument("--nwires", type=int, default=0, help="override the workload's wire count")
    ap.add_argument("--acc-steps", type=int, default=4000,
                    help="time steps of the accuracy check (the workload's duration, at most "
                         "this; 0 skips it)")
    ap.add_argument("--rate", type=float, default=2000.0, help="c4: requests per second")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="c4: stream length served in real time by the split form")
    ap.add_argument("--plain-serve-seconds", type=float, default=15.0,
                    help="c4: stream length served in real time by the plain form")
    ap.add_argument("--capacity-requests", type=int, default=24000,
                    help="c4: backlog of the saturated capacity runs (both forms)")
    ap.add_argument("--no-serve", action="store_true", help="c4: skip the serving runs")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch each bench step eagerly instead of replaying its CUDA graph")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-baseline", action="store_true",
                    help="skip timing the reference's own Numba path")
    return ap.parse_args()


def c4_stream(rank, seconds, rate=2000.0, chunk=50):
    """The configuration-4 request stream of one rank (seeded Poisson arrivals)."""
    from pulsesuite_b200 import serve

    return serve.poisson_stream(rate=rate, seconds=seconds, seed=4 + 1000 * rank, chunk=chunk)


def make_workload(name, rank, nwires):
    from pulsesuite_b200 import workloads

    if name == "c4":
        # the request mix of the serving stream as a resident batch of wires:
        # the first `nwires` requests of the rank's stream, each its own Nk,
        # pulse, detuning, FWHM and T2.  16384 is about the server's slot
        # capacity (default_capacity: 15360 slots), i.e. the resident load of
        # a saturated server; fewer leave the Nk-1024 class too few CTAs to
        # fill the GPU, and a step is then the latency of its longest CTA
        from pulsesuite_b200 import abi, serve
        from pulsesuite_b200 import grid as pgrid

        n = nwires or 16384
        reqs = c4_stream(rank, seconds=1.2 * n / 2000.0 + 1.0)[:n]
        grids = [pgrid.wire_grid(nk) for nk in serve.C4_NKS]
        w = np.concatenate([serve.wire_record(r, grids[serve.C4_NKS.index(r.nk)],
                                              table=serve.C4_NKS.index(r.nk)) for r in reqs])
        assert w.dtype == abi.WIRE_DTYPE
        return workloads.Workload(f"c4 request mix: {len(w)} resident solves", grids, w, 4000,
                                  1e-15)
    kw = {"seed": 1 + 1000 * rank + {"c1": 0, "c2": 1, "c3": 2}[name]}
    if nwires:
        kw["nwires"] = nwires
    return workloads.CONFIGS[name](**kw)


def config_for(a, wl, world):
    """The line's `config`, identical in both arms (ours and --impl reference)."""
    cfg = {"workload": WORKLOAD_NAMES[a.workload], "resident_batch": wl.name,
           "wires_per_gpu": int(len(wl.wires)), "wire_k_per_time_step": int(wl.units_per_step),
           "time_steps_per_bench_step": int(a.chunk),
           "l2": "256 MiB write between timed steps (outside the events)",
           "parallelism": f"wires sharded, {world} independent GPU(s)"}
    if a.workload == "c4":
        cfg["serving"] = {"rate_per_s": a.rate, "seconds": a.serve_seconds,
                          "capacity_requests": a.capacity_requests, "tick_steps": 50,
                          "hbm_budget_GB": 150}
    return cfg


WORKLOAD_NAMES = {
    "c1": "c1: 1024 wires, Nk U[64,512] rounded to 32, pulse area U[0.1pi,2pi], detuning "
          "U[-50,50] meV, FWHM U[20,200] fs, T2 U[50,300] fs, 3000 x 1 fs RK4",
    "c2": "c2: 16384 wires, Nk 512, statically screened (eps(q; n1D) every RHS), pulse area "
          "U[0.2pi,1.5pi], 2000 x 1 fs RK4",
    "c3": "c3: 65536 wires (256x256 sites), Nk 256, pump 30 fs + probe 15 fs (delay U[0,200] "
          "fs, phase U[0,2pi)), T2 100 fs, 4000 x 0.5 fs RK4",
    "c4": "c4: Poisson 2000 requests/s for 60 s, Nk in {64,128,256,512,1024} "
          "p={.3,.3,.2,.15,.05}, 1-4 ps at 1 fs, parameters as c1, 150 GB HBM budget",
}


# ---------------------------------------------------------------------------
# pstd: the PSTD caller's step of all its wires (rhoPJ.QuantumWire's loop of
# QWCalculator calls, rhoPJ.py:311-348) on the full Nk x Nk state with every
# many-body term.
# ---------------------------------------------------------------------------
PSTD_QW = """{L}     # L
5e-9       # Delta0
1.5        # gap
0.07       # me
0.45       # mh
100e-3     # HO
5e12       # gam_e
5e12       # gam_h
5e12       # gam_eh
9.1        # epsr
36e-3      # Oph
3e-3       # Gph
2000000.0  # Edc
1000000    # jmax
20000      # ntmax
"""
# Optics Excitons EHs Screened Phonon DCTrans LF FreePot DiagDph OffDiagDph
# Recomb PLSpec ignorewire Xqwparams LorentzDelta
PSTD_MB = "1\n1\n1\n1\n1\n1\n1\n0\n1\n1\n1\n0\n0\n0\n0\n"
PSTD_L, PSTD_NRR, PSTD_DT, PSTD_E0 = 1e-7, 64, 1e-17, 1e8
PSTD_METRIC = "full-matrix wire-steps/s (QWCalculator steps of all wires per Maxwell step)"


def pstd_config(nw):
    return {"workload": f"pstd: one Maxwell step of {nw} quantum wires (rhoPJ.QuantumWire's "
                        "QWCalculator loop), L 100 nm (Nk 114), 64-point propagation grid, "
                        "full Nk x Nk state, screened, LF, DiagDph OffDiagDph EHs Phonon "
                        "Recomb DCTrans (Edc 2 MV/m), dt 10 as",
            "wires_per_gpu": int(nw), "time_steps_per_bench_step": 1,
            "l2": "256 MiB write between timed steps (outside the events)",
            "parallelism": "wires sharded, independent GPU(s)"}


def pstd_solver(path, nw):
    from pulsesuite_b200 import SBEs

    os.makedirs(os.path.join(path, "params"), exist_ok=True)
    with open(os.path.join(path, "params", "qw.params"), "w") as f:
        f.write(PSTD_QW.format(L=PSTD_L))
    with open(os.path.join(path, "params", "mb.params"), "w") as f:
        f.write(PSTD_MB)
    cwd = os.getcwd()
    os.chdir(path)
    try:
        return SBEs.SBESolver(None, np.linspace(-5e-8, 5e-8, PSTD_NRR), 0.0, 1e7, 800e-9, nw,
                              True)
    finally:
        os.chdir(cwd)


def pstd_fields(i):
    """The propagation-space fields along the wire at step i: a Gaussian
    profile (every q on the wire) under a carrier at 1.55 eV."""
    rr = np.linspace(-5e-8, 5e-8, PSTD_NRR)
    prof = np.exp(-((rr / 3e-8) ** 2))
    E = PSTD_E0 * np.cos(2.35e15 * i * PSTD_DT)
    return rr, [(0.3 * E * prof * (rr / 3e-8)).astype(complex), (E * prof).astype(complex),
                (0.2 * E * prof).astype(complex), np.zeros(PSTD_NRR, complex)]


def pstd_reference_sample(threads, nsteps=2):
    """The reference's own QWCalculator on the host cores, one wire of the
    same configuration: (wire-steps/s, the cpu_baseline record)."""
    from oracle import numba_ref

    if not numba_ref.available():
        return None, {"unavailable": "reference not installed under baseline/_ref"}
    import platform

    R = numba_ref.load(threads=threads)
    sec, nk = numba_ref.qwcalc_seconds_per_wire_step(R, PSTD_QW.format(L=PSTD_L), PSTD_MB,
                                                     nrr=PSTD_NRR, nsteps=nsteps, E0=PSTD_E0)
    return 1.0 / sec, {"value": 1.0 / sec, "unit": "wire-steps/s", "cores": int(R.threads),
                       "kind": "reference", "cpu": platform.processor() or platform.machine(),
                       "sample": f"reference SBESolver.QWCalculator, one wire, Nk {nk}, "
                                 f"mean of {nsteps} calls after one compiling call: "
                                 f"{sec * 1e3:.1f} ms per wire-step"}


def run_pstd(a):
    """One bench step = one Maxwell step of all the rank's wires (one
    QWCalculator step per wire).  value: the batched full step
    (psb_full_step_batch_f64 + psb_full_sources_batch_f64) with the
    wire-space fields resident on the device, CUDA events, max over ranks;
    e2e: SBESolver.QWCalculatorAll with host fields in and host sources out
    (Prop2QW / QW2Prop on the host, copies each way); per_wire_loop: the
    reference's calling pattern, one QWCalculator call per wire.  The
    reference arm times the reference's own QWCalculator on the host cores."""
    import tempfile

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    nw = a.nwires or 64
    threads = os.cpu_count() or 1
    if a.impl == "reference":
        if rank != 0:
            return
        for _ in range(max(1, a.warmup)):
            pstd_reference_sample(threads, nsteps=1)
        t0 = time.perf_counter()
        vals = [pstd_reference_sample(threads, nsteps=1) for _ in range(a.steps)]
        wall = time.perf_counter() - t0
        if vals[-1][0] is None:
            print(json.dumps({"impl": "reference", "unavailable": vals[-1][1]["unavailable"]}))
            return
        v = float(np.mean([x[0] for x in vals]))
        cb = dict(vals[-1][1])
        cb["value"] = v
        print(json.dumps({
            "impl": "reference", "metric": PSTD_METRIC, "value": v, "unit": "wire-steps/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": wall * 1e3 / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (deterministic fields)",
            "config": pstd_config(nw),
            "form": "reference SBESolver.QWCalculator (Python + Numba), one wire per bench step",
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "wire-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return

    import torch
    import torch.distributed as dist

    from pulsesuite_b200 import _lib, device, wirespace

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    tmp = tempfile.mkdtemp(prefix="psb_pstd_")
    s = pstd_solver(os.path.join(tmp, "a"), nw)
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def maxwell_step(solver, i, batched=True):
        rr, f = pstd_fields(i)
        o = [np.zeros((PSTD_NRR, nw), complex) for _ in range(4)]
        if batched:
            solver.QWCalculatorAll(*f, rr, None, PSTD_DT, *o, [False], [False])
        else:
            for w in range(nw):
                ow = [np.zeros(PSTD_NRR, complex) for _ in range(4)]
                solver.QWCalculator(*f, rr, None, PSTD_DT, w + 1, *ow, [False], [False])
                for x, y in zip(o, ow):
                    x[:, w] = y
        return o

    for i in range(max(1, a.warmup)):
        maxwell_step(s, i)
    # device-resident inputs: the wire-space fields of one step
    rr, f = pstd_fields(a.warmup)
    wf = wirespace.prop2qw_rows(rr, np.stack(f), s.r, s.window)
    fd, wpd = s._full_batch_inputs(0, np.ascontiguousarray(np.broadcast_to(wf[:3], (nw, 3, s.Nr))),
                                   PSTD_DT)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(a.steps)]
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    with Clocks(local) as clk:
        for k in range(a.steps):
            flush.fill_(float(k))
            evs[k][0].record(stream)
            s._full_launch_batch(0, fd, wpd, PSTD_DT)
            evs[k][1].record(stream)
        torch.cuda.synchronize()
    total_ms = float(sum(e0.elapsed_time(e1) for e0, e1 in evs))
    # end to end through the public API
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(a.steps):
        maxwell_step(s, a.warmup + 1 + k)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    # the per-wire calling pattern of the reference's caller, on a second solver
    b = pstd_solver(os.path.join(tmp, "b"), nw)
    maxwell_step(b, 0, batched=False)
    kl = min(a.steps, 3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(kl):
        maxwell_step(b, 1 + k, batched=False)
    torch.cuda.synchronize()
    loop_s = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([total_ms, e2e_s, loop_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, e2e_s, loop_s = (float(x) for x in t.tolist())
        dist.barrier()
    value = nw * a.steps * world / (total_ms * 1e-3)
    nk, nr = s.Nk, s.Nr
    mb = s.full["mb"]
    # screen; meh, calch; gamma, offd, offp; derivs; x3, rates, relax;
    # shift, rows, cols; leapfrog; sources
    launches = 1 + 2 + 3 + 1 + 3 + 3 + 1 + 1
    assert mb is not None and s.Screened and s.LF
    fp64 = fp64_peak_tflops(torch, _lib, device)
    ach = 96.0 * nk ** 3 * nw / (total_ms / a.steps * 1e-3) / 1e12
    line = {
        "metric": PSTD_METRIC, "value": value, "unit": "wire-steps/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_ms / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (deterministic fields)", "config": pstd_config(nw),
        "e2e": {"value": nw * a.steps * world / e2e_s, "unit": "wire-steps/s",
                "h2d_bytes_per_step": nw * (3 * nr * 16 + 4 * 8),
                "d2h_bytes_per_step": nw * (5 * nr * 16 + 2 * nk * 16),
                "api": "pulsesuite_b200.SBEs.SBESolver.QWCalculatorAll (host arrays, "
                       "Prop2QW / QW2Prop on the host)",
                "ms_per_step": e2e_s * 1e3 / a.steps},
        "per_wire_loop": {"value": nw * kl * world / loop_s, "unit": "wire-steps/s",
                          "api": "SBESolver.QWCalculator once per wire (rhoPJ.py:311-348)",
                          "ms_per_step": loop_s * 1e3 / kl},
        "roofline": {"bound": "fp64", "achieved": ach, "peak": fp64, "unit": "TFLOP/s",
                     "frac": ach / fp64, "traffic": None,
                     "work": "96 Nk^3 flops per wire-step: the 12 complex Nk x Nk x Nk "
                             "products of dpdt/dCdt/dDdt; the step's other O(Nk^3) kernels "
                             "(exchange sums, dephasing, scattering, DC shift, source sums) "
                             "count as overhead",
                     "peak_source": "measured in this run: psb_probe_fp64_fma"},
        "gpu_launches": launches * a.steps,
        "clocks": clk.summary(),
    }
    if rank == 0 and not a.no_cpu_baseline:
        try:
            line["cpu_baseline"] = pstd_reference_sample(threads)[1]
        except Exception as ex:
            line["cpu_baseline"] = {"unavailable": f"{type(ex).__name__}: {ex}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Clock sampling during the timed region.
# ---------------------------------------------------------------------------
class Clocks:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is None:
            return
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        self.rows = [r.split(",") for r in out.strip().splitlines() if r.strip()]

    def summary(self):
        if self.proc is None or not getattr(self, "rows", None):
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, r[4:8]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# CPU baselines.
# ---------------------------------------------------------------------------
def cpu_baseline(wl, seconds, threads):
    """The oracle (OpenMP C restatement of the reference's path, the same
    O(Nk^2) diagonal arithmetic as the GPU kernels) on a sample of the
    workload's wires, all host threads."""
    from scipy.constants import hbar

    from oracle import oracle as orc
    from pulsesuite_b200 import grid as pgrid

    rng = np.random.default_rng(7)
    blocks = [orc.grid_tables(g, screened=wl.screened) for g in wl.grids]
    tables, tabdata = pgrid.pack_tables(wl.grids, blocks, screened=wl.screened)

    def run(nw, nsteps):
        idx = rng.choice(len(wl.wires), size=min(nw, len(wl.wires)), replace=False)
        w = wl.wires[idx].copy()
        nks = tables["nk"][w["table"]].astype(np.int64)
        w["off"] = np.concatenate([[0], np.cumsum(nks)[:-1]])
        y = np.zeros(4 * int(nks.sum()))
        t0 = time.perf_counter()
        orc.rk4(tables, tabdata, w, y, nsteps, wl.dt, hbar, nthreads=threads)
        el = time.perf_counter() - t0
        return float(nks.sum()) * nsteps / el, el, len(w)

    # calibrate with a short run, then size the sample to ~`seconds`
    rate, el, _ = run(2 * threads, 4)
    units_per_wire_step = float(np.mean(wl.nks))
    budget = rate * seconds / units_per_wire_step  # wire*steps that fit the budget
    nw = int(max(threads, min(len(wl.wires), budget / 20)))
    nsteps = int(max(4, min(400, budget / nw)))
    rate, el, nw = run(nw, nsteps)
    return {"value": rate, "unit": "wire*k*steps/s", "cores": threads, "kind": "port",
            "sample": f"{nw} wires drawn from the workload x {nsteps} RK4 steps "
                      f"({el:.1f} s, OpenMP over wires)"}


def cpu_baseline_reference(wl, threads, measure_nks=(64, 128, 256)):
    """The reference's own Numba CPU path (baseline/_ref; full Nk x Nk
    CalcH + dpdt/dCdt/dDdt integrated by rk4_dpc, Numba threads inside the
    kernels), timed for one RK4 step of one wire at each measured Nk and
    weighted by the workload's wires: wire*k*steps/s = sum Nk / sum t(Nk).
    Grids above the largest measured one are extrapolated with the power
    law through the two largest measurements (the reference is O(Nk^3) per
    right-hand side).  Screening (c2) is not included in the timed RHS and
    the two-pulse drive (c3) is timed as one pulse (same cost)."""
    from oracle import numba_ref

    if not numba_ref.available():
        return {"unavailable": "reference not installed under baseline/_ref"}
    import platform

    t0 = time.perf_counter()
    R = numba_ref.load(threads=threads)
    load_s = time.perf_counter() - t0
    from pulsesuite_b200 import abi
    from pulsesuite_b200 import grid as pgrid

    nks_all = wl.nks
    present = sorted(set(int(n) for n in nks_all))
    meas = sorted(set([n for n in present if n <= max(measure_nks)] +
                      [n for n in measure_nks if n <= max(present)]))
    per = {}
    for nk in meas:
        g = pgrid.wire_grid(nk)
        w = np.zeros(1, dtype=abi.WIRE_DTYPE)
        src = wl.wires[int(np.argmin(np.abs(nks_all - nk)))]
        w[0] = src
        w["npulse"] = 1
        per[nk] = numba_ref.seconds_per_step(R, g, w[0], wl.dt, nsteps=2)
    ms = sorted(per)
    if len(ms) >= 2:
        n1, n2 = ms[-2], ms[-1]
        expo = float(np.log(per[n2] / per[n1]) / np.log(n2 / n1))
    else:
        expo = 3.0

    def t_of(nk):
        if nk in per:
            return per[nk]
        ref = min(ms, key=lambda m: abs(np.log(m / nk)))
        return per[ref] * (nk / ref) ** expo

    total_t = float(sum(t_of(int(n)) for n in nks_all))
    value = float(nks_all.sum()) / total_t
    extrap = sorted(set(int(n) for n in nks_all) - set(per))
    return {"value": value, "unit": "wire*k*steps/s", "cores": int(R.threads),
            "kind": "reference", "cpu": platform.processor() or platform.machine(),
            "sample": "reference SBEs._CalcH_jit (recompiled serial, parallel build wrong "
                      "under numba 0.65) + _dpdt/_dCdt/_dDdt_jit + integrator.rk4_dpc, "
                      "mean of two RK4 steps of one wire per measured Nk "
                      + ", ".join(f"{k}: {v * 1e3:.1f} ms" for k, v in sorted(per.items()))
                      + (f"; Nk {extrap} extrapolated as Nk^{expo:.2f}" if extrap else ""),
            "extrapolated": bool(extrap), "import_and_jit_s": load_s}


# ---------------------------------------------------------------------------
def fp64_peak_tflops(torch, _lib, device):
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    sink = torch.zeros(sms * 8, dtype=torch.float64, device="cuda")
    import ctypes

    ms = ctypes.c_float(0.0)
    best = 0.0
    iters = 20000
    for _ in range(3):
        _lib.call("psb_probe_fp64_fma", sms * 8, iters, device.ptr(sink), ctypes.byref(ms),
                  device.stream_ptr())
        flops = 2.0 * 8 * iters * sms * 8 * 256
        best = max(best, flops / (ms.value * 1e-3) / 1e12)
    return best


def measured_bf16_peak():
    """Dense bf16 peak of this pool's B200s (driver-measured cuBLAS burst)."""
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            v = float(json.load(f)["bf16_tflops"])
        return v, "MEASURED_PEAKS.json bf16_tflops (cuBLAS burst), of measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback 1.59 PFLOP/s (no MEASURED_PEAKS.json)"


def split_accuracy(wl, nsteps, stream):
    """Per-wire error of the split form against the plain FP64 form (which
    matches the FP64 oracle to <= 1e-10) on the same workload from the same
    zero state, max and median over wires:
    P: max_t |P - P_ref| / max_t |P_ref|;
    n: max_k |n - n_ref| / max_k |n_ref| of the final n_e and n_h;
    p: max_k |p - p_ref| of the final state over the wire's peak p scale
    max_t |P_ref| / (|pscale| Nk) (p itself may have dephased to ~1e-20 by
    the end, below the rounding floor of its peak, so it is not a scale)."""
    import torch

    from pulsesuite_b200.batch import WireBatch

    out = {}
    for form in ("split", "plain"):
        bb = WireBatch(wl.grids, wl.wires, screened=wl.screened, p_cap=nsteps, form=form)
        bb.rk4(nsteps, wl.dt, p_stride=1, stream=stream)
        torch.cuda.synchronize()
        out[form] = (bb.P[:bb.nw * nsteps].view(bb.nw, nsteps, 2).clone(), bb.y.clone(),
                     [bb.wire_slice(i) for i in range(bb.nw)])
        del bb
    Ps, ys, sl = out["split"]
    Pp, yp, _ = out["plain"]
    dP = torch.linalg.vector_norm(Ps - Pp, dim=2).amax(dim=1)
    refP = torch.linalg.vector_norm(Pp, dim=2).amax(dim=1)
    errP = (dP / refP.clamp_min(1e-300)).cpu().numpy()
    refP = refP.cpu().numpy()
    d = ys - yp
    dpk = torch.sqrt(d[:, 0] ** 2 + d[:, 1] ** 2).cpu().numpy()
    dn, rn = d[:, 2:].abs().cpu().numpy(), yp[:, 2:].abs().cpu().numpy()
    errN = np.zeros(len(sl))
    errp = np.zeros(len(sl))
    nks = wl.nks
    for i, r in enumerate(sl):
        errN[i] = max(dn[r, c].max() / max(rn[r, c].max(), 1e-300) for c in range(2))
        pk = refP[i] / max(abs(float(wl.wires["pscale"][i])) * nks[i], 1e-300)
        errp[i] = dpk[r].max() / max(pk, 1e-300)
    return {"vs": "plain FP64 form (<= 1e-10 from the FP64 oracle)", "time_steps": nsteps,
            "P_rel_err_max": float(errP.max()), "P_rel_err_median": float(np.median(errP)),
            "n_rel_err_max": float(errN.max()), "n_rel_err_median": float(np.median(errN)),
            "p_err_vs_peak_max": float(errp.max()),
            "p_err_vs_peak_median": float(np.median(errp))}


def step_traffic(b, S):
    """Estimated DRAM bytes of one bench step (see DRAM_* above)."""
    if b.form == "plain":
        return DRAM_PLAIN_PER_ELEMENT * b.n_state
    from pulsesuite_b200 import _lib, abi

    lib = _lib.load()
    nks = b.h_tables["nk"]
    total = 0.0
    for wg, groups, ng, nkmax in b.split_launches:
        g = groups.cpu().numpy().view(abi.SPLIT_GROUP_DTYPE)
        elements = float(np.sum(g["nw"].astype(np.float64) * nks[g["table"]]))
        if nkmax <= int(lib.psb_split_max_nk_resident(wg)):
            total += DRAM_SPLIT_RES_PER_ELEMENT * elements
        else:
            total += DRAM_SPLIT_WS_PER_ELEMENT_STEP * elements * S
    # per-wire matrices (screened or distinct): the stage state is always in
    # the workspace
    for wg, groups, ng, nkmax, tflags in b.wire_launches:
        g = groups.cpu().numpy().view(abi.SPLIT_GROUP_DTYPE)
        elements = float(np.sum(g["nw"].astype(np.float64) * nks[g["table"]]))
        total += DRAM_SPLIT_WS_PER_ELEMENT_STEP * elements * S
    return total


def oracle_accuracy(wl, nsteps, stream, nsample=16):
    """Plain-form error against the FP64 oracle on a sample of wires over
    `nsteps` (the check used where the split form does not apply)."""
    import torch
    from scipy.constants import hbar

    from oracle import oracle as orc
    from pulsesuite_b200 import grid as pgrid
    from pulsesuite_b200.batch import WireBatch

    rng = np.random.default_rng(11)
    idx = np.sort(rng.choice(len(wl.wires), size=min(nsample, len(wl.wires)), replace=False))
    w = wl.wires[idx].copy()
    b = WireBatch(wl.grids, w, screened=wl.screened, p_cap=nsteps, form="plain")
    b.rk4(nsteps, wl.dt, stream=stream)
    torch.cuda.synchronize()
    blocks = [orc.grid_tables(g, screened=wl.screened) for g in wl.grids]
    tables, tabdata = pgrid.pack_tables(wl.grids, blocks, screened=wl.screened)
    ww = w.copy()
    nks = tables["nk"][ww["table"]].astype(np.int64)
    ww["off"] = np.concatenate([[0], np.cumsum(nks)[:-1]])
    ww["p_off"] = np.arange(len(ww)) * nsteps
    yo = np.zeros(4 * int(nks.sum()))
    Po = orc.rk4(tables, tabdata, ww, yo, nsteps, wl.dt, hbar, p_stride=1, p_cap=nsteps,
                 nthreads=os.cpu_count() or 1).reshape(len(ww), nsteps)
    yo = yo.reshape(-1, 4)
    y = b.state()
    eP, ep, en = [], [], []
    for i in range(len(ww)):
        sl = b.wire_slice(i)
        rP = b.records(i)
        eP.append(np.max(np.abs(rP - Po[i])) / max(np.max(np.abs(Po[i])), 1e-300))
        pr, po = y[sl, 0] + 1j * y[sl, 1], yo[sl, 0] + 1j * yo[sl, 1]
        ep.append(np.max(np.abs(pr - po)) / max(np.max(np.abs(po)), 1e-300))
        en.append(max(np.max(np.abs(y[sl, c] - yo[sl, c])) / max(np.max(np.abs(yo[sl, c])), 1e-300)
                      for c in (2, 3)))
    return {"vs": "FP64 oracle (CPU restatement pinned to the reference's goldens)",
            "form": "plain", "time_steps": nsteps, "wires": int(len(ww)),
            "P_rel_err_max": float(np.max(eP)), "p_rel_err_max": float(np.max(ep)),
            "n_rel_err_max": float(np.max(en))}


def timed_steps(b, S, dt, K, W, stream, flush, world, graph=True):
    """W warm-up bench steps, then K bench steps of S time steps each, every
    one bracketed by CUDA events on `stream` with an L2 flush between them
    (outside the events); total device ms, max over ranks.  With `graph` a
    bench step is one replay of the CUDA graph of the batch's rk4 call."""
    import torch
    import torch.distributed as dist

    if graph:
        g = b.capture(S, dt, p_stride=1)

        def step():
            g.replay()
    else:
        def step():
            b.rk4(S, dt, p_stride=1, stream=stream)
    for _ in range(W):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(K)]
    torch.cuda.synchronize()
    for i in range(K):
        flush.fill_(float(i))
        evs[i][0].record(stream)
        step()
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    total_ms = float(sum(e0.elapsed_time(e1) for e0, e1 in evs))
    if world > 1:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    return total_ms


def pipelined_e2e(b, wl, S, K, stream, world):
    """End to end through the public API: every bench step copies its input
    state from pinned host memory and reads its P(t) records and final state
    back to pinned host memory; the copies run on their own streams and
    overlap the neighbouring steps' compute, as a caller streaming
    independent batches through the API would run them:
      upload stream:    H2D input(i+1) -> staging
      download stream:  D2H snapshot(i) -> host(i % 2)
      compute:      staging -> y, rk4, y/P -> snapshot(i % 2)
    The timed region spans all K steps, from before the first upload to after
    the last download; it includes two device-to-device staging copies per
    step (not counted in the host<->device bytes) and no L2 flush."""
    import torch
    import torch.distributed as dist

    y_host = torch.zeros((b.n_state, 4), dtype=torch.float64).pin_memory()
    y_out = [torch.empty_like(y_host).pin_memory() for _ in range(2)]
    P_out = [torch.empty(tuple(b.P.shape), dtype=torch.float64).pin_memory() for _ in range(2)]
    y_stage = torch.empty_like(b.y)
    y_snap = [torch.empty_like(b.y) for _ in range(2)]
    P_snap = [torch.empty_like(b.P) for _ in range(2)]
    cs_up, cs_dn = torch.cuda.Stream(), torch.cuda.Stream()
    ev = lambda: torch.cuda.Event()  # noqa: E731
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    cs_up.wait_event(e0)
    cs_dn.wait_event(e0)
    staged = ev()
    with torch.cuda.stream(cs_up):
        y_stage.copy_(y_host, non_blocking=True)
    staged.record(cs_up)
    out_done = [None, None]
    for i in range(K):
        stream.wait_event(staged)
        b.y.copy_(y_stage)
        consumed = ev()
        consumed.record(stream)
        b.rk4(S, wl.dt, p_stride=1, stream=stream)
        j = i % 2
        if out_done[j] is not None:
            stream.wait_event(out_done[j])  # host buffer j and its snapshot are free
        y_snap[j].copy_(b.y)
        P_snap[j].copy_(b.P)
        snapped = ev()
        snapped.record(stream)
        if i + 1 < K:
            with torch.cuda.stream(cs_up):
                cs_up.wait_event(consumed)
                y_stage.copy_(y_host, non_blocking=True)
                staged = ev()
                staged.record(cs_up)
        with torch.cuda.stream(cs_dn):
            cs_dn.wait_event(snapped)
            y_out[j].copy_(y_snap[j], non_blocking=True)
            P_out[j].copy_(P_snap[j], non_blocking=True)
            out_done[j] = ev()
            out_done[j].record(cs_dn)
    for d in out_done:
        if d is not None:
            stream.wait_event(d)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    return e2e_ms, y_host.numel() * 8, (P_out[0].numel() + y_out[0].numel()) * 8


CAP_INFLIGHT = 8  # ticks a lane may queue in the saturated-capacity runs


def serve_section(a, rank, world):
    """Configuration 4 through the serving API: saturated capacity of both
    forms on the same backlog (the first `capacity_requests` requests of the
    rank's stream, all queued at once), and the Poisson stream served in real
    time (split form: `serve_seconds`; plain form: `plain_serve_seconds`)."""
    import torch
    import torch.distributed as dist

    from pulsesuite_b200 import serve

    chunk = 50
    warm = serve.poisson_stream(rate=200.0, seconds=0.1, seed=99, chunk=chunk)
    sat = c4_stream(rank, seconds=1.1 * a.capacity_requests / a.rate + 1.0, rate=a.rate,
                    chunk=chunk)[:a.capacity_requests]
    out = {"capacity": {}, "realtime": {}}
    # the capacity runs queue up to 8 ticks per lane (throughput: the host
    # loop stays ahead of the GPU while the short ticks of the small grids
    # drain; 8 measured ~9 % above 4, within the run-to-run spread); the
    # real-time runs keep the default 2 (latency: a new request waits behind
    # fewer queued ticks)
    # the saturated capacity varies by ~10 % from run to run (host loop and
    # stream interleaving): the split form's is the median of three runs of
    # the same backlog, all three listed; the plain form's (12 s a run) one
    for form, reps in (("split", 3), ("plain", 1)):
        srv = serve.Server(form=form, chunk=chunk, max_inflight_ticks=CAP_INFLIGHT)
        srv.run(warm, realtime=False)
        runs = []
        for _ in range(reps):
            srv.reset_counters()
            res = srv.run(sat, realtime=False)
            ok = all(r.status == 0 for r in res)
            runs.append({"value": srv.throughput(), "seconds": srv.elapsed,
                         "requests": len(res), "ticks": srv.tick_count,
                         "ticks_in_flight_per_lane": CAP_INFLIGHT, "h2d_bytes": srv.h2d_bytes,
                         "d2h_bytes": srv.d2h_bytes, "status_ok": ok})
        best = sorted(runs, key=lambda r: r["value"])[len(runs) // 2]
        out["capacity"][form] = dict(best, runs=[r["value"] for r in runs],
                                     status_ok=all(r["status_ok"] for r in runs))
        del srv
        torch.cuda.synchronize()
    for form, secs in (("split", a.serve_seconds), ("plain", a.plain_serve_seconds)):
        if secs <= 0:
            continue
        reqs = c4_stream(rank, seconds=secs, rate=a.rate, chunk=chunk)
        srv = serve.Server(form=form, chunk=chunk)
        srv.run(warm, realtime=False)
        res = srv.run(reqs, realtime=True)
        lat = srv.latency_percentiles((50, 99))
        out["realtime"][form] = {"seconds_of_stream": secs, "requests": len(res),
                                 "throughput": srv.throughput(), "p50_s": lat.get(50),
                                 "p99_s": lat.get(99),
                                 "status_ok": all(r.status == 0 for r in res)}
        del srv
        torch.cuda.synchronize()
    if world > 1:
        for form in ("split", "plain"):
            t = torch.tensor([out["capacity"][form]["value"]], device="cuda",
                             dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
            out["capacity"][form]["value"] = float(t.item())
    c = out["capacity"]
    c["split_over_plain"] = c["split"]["value"] / c["plain"]["value"]
    return out


def run_ours(a):
    import torch
    import torch.distributed as dist

    from pulsesuite_b200 import _lib, device
    from pulsesuite_b200.batch import WireBatch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    wl = make_workload(a.workload, rank, a.nwires)
    form, form_note = a.form, None
    if wl.screened and form == "split":
        form_note = ("screened: per-wire Coulomb matrices V/eps(q; n1D) rebuilt every RK "
                     "stage, psb_rk4_split_wire")
    S = a.chunk
    b = WireBatch(wl.grids, wl.wires, screened=wl.screened, p_cap=S, form=form)
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    units = wl.units_per_step * S

    with Clocks(local) as clk:
        total_ms = timed_steps(b, S, wl.dt, a.steps, a.warmup, stream, flush, world,
                               graph=not a.no_graph)
    value = units * a.steps * world / (total_ms * 1e-3)
    status = b.wires()["status"]
    plain = None
    if form == "split" and not a.no_plain:
        bp = WireBatch(wl.grids, wl.wires, screened=wl.screened, p_cap=S, form="plain")
        pms = timed_steps(bp, S, wl.dt, a.steps, a.warmup, stream, flush, world,
                          graph=not a.no_graph)
        pval = units * a.steps * world / (pms * 1e-3)
        fp64 = fp64_peak_tflops(torch, _lib, device)
        pach = wl.flops_per_step() * S / (pms / a.steps * 1e-3) / 1e12
        plain = {"value": pval, "ms_per_step": pms / a.steps, "split_over_plain": value / pval,
                 "gpu_launches": a.steps * bp.launches_per_call,
                 "roofline": {"bound": "fp64", "achieved": pach, "peak": fp64,
                              "unit": "TFLOP/s", "frac": pach / fp64,
                              "peak_source": "measured in this run: psb_probe_fp64_fma"}}
        del bp
    accuracy = None
    if a.acc_steps > 0:
        if form == "split" and not a.no_plain:
            # the workload's own duration, bounded (at most ~2e10 wire*k*steps)
            # a sample of at most 4096 wires over the workload's duration
            # (at most ~2e10 wire*k*steps), so the check stays a few seconds
            acc_wl = wl
            if len(wl.wires) > 4096:
                from pulsesuite_b200 import workloads

                acc_wl = workloads.Workload(wl.name + " (first 4096 wires)", wl.grids,
                                            wl.wires[:4096], wl.nsteps, wl.dt, wl.screened)
            n_acc = min(acc_wl.nsteps, a.acc_steps, max(50, int(2e10 // acc_wl.units_per_step)))
            accuracy = split_accuracy(acc_wl, n_acc, stream)
            accuracy["wires"] = int(len(acc_wl.wires))
        elif form == "plain" and rank == 0:
            accuracy = oracle_accuracy(wl, min(wl.nsteps, a.acc_steps, 300), stream)

    serving = None
    if a.workload == "c4" and not a.no_serve:
        serving = serve_section(a, rank, world)
        cs = serving["capacity"]["split" if form == "split" else "plain"]
        e2e = {"value": cs["value"], "unit": "wire*k*steps/s",
               "h2d_bytes_per_step": cs["h2d_bytes"] / max(1, cs["ticks"]),
               "d2h_bytes_per_step": cs["d2h_bytes"] / max(1, cs["ticks"]),
               "api": "pulsesuite_b200.serve.Server.run (saturated backlog)",
               "step": "one server tick (one launch of one size class)",
               "requests": cs["requests"]}
    else:
        e2e_ms, h2d, d2h = pipelined_e2e(b, wl, S, a.steps, stream, world)
        e2e = {"value": units * a.steps * world / (e2e_ms * 1e-3), "unit": "wire*k*steps/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "api": "WireBatch.rk4 with pinned host state in and P(t) + state out"}

    avg_launch_ms = total_ms / a.steps
    if form == "plain":
        peak = fp64_peak_tflops(torch, _lib, device)
        peak_source = "measured in this run: psb_probe_fp64_fma (FMA loop)"
        bound, unit = "fp64", "TFLOP/s"
        flops_launch = wl.flops_per_step() * S
    else:
        # the split algorithm's tensor-core work: 6 int8 digit products x 4
        # columns x Nk MACs (2 ops) per element and stage, 4 stages per step
        # (unpadded grid)
        flops_launch = float(np.sum(wl.nks.astype(np.float64) ** 2)) * 192.0 * S
        peak, peak_source = measured_bf16_peak()
        # dense int8 tensor rate is twice the bf16 rate on B200
        peak, peak_source = 2.0 * peak, "2 x " + peak_source
        bound, unit = "tensor", "TOP/s"
    achieved = flops_launch / (avg_launch_ms * 1e-3) / 1e12
    traffic = step_traffic(b, S)

    line = {
        "metric": METRIC,
        "value": value,
        "unit": "wire*k*steps/s",
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": total_ms / a.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if form == "plain" else "int8x3digits+s32acc+f64",
        "data": "synthetic (seeded configuration draws)",
        "config": config_for(a, wl, world),
        "form": form,
        "e2e": e2e,
        "roofline": {"bound": bound, "achieved": achieved, "peak": peak, "unit": unit,
                     "frac": achieved / peak, "traffic": traffic,
                     "traffic_source": TRAFFIC_SOURCE, "peak_source": peak_source,
                     "flops_per_launch": flops_launch},
        "gpu_launches": a.steps * b.launches_per_call,
        "launch": "eager" if a.no_graph else "CUDA graph replay per bench step",
        "plain": plain,
        "accuracy": accuracy,
        "serving": serving,
        "clocks": clk.summary(),
        "wire_status_ok": bool((status == 0).all()),
    }
    if form_note:
        line["form_note"] = form_note
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        threads = os.cpu_count() or 1
        line["cpu_baseline"] = cpu_baseline(wl, a.cpu_seconds, threads)
        if not a.no_reference_baseline:
            try:
                line["cpu_baseline_reference"] = cpu_baseline_reference(wl, threads)
            except Exception as ex:  # reported, not fatal: the baseline is informational
                line["cpu_baseline_reference"] = {"unavailable": f"{type(ex).__name__}: {ex}"}
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference(a):
    """The reference arm: the CPU implementation of the path on the host
    cores, on the same workload and `config` as our arm.  The reference
    itself is Python/Numba with an O(Nk^3) full-matrix RHS; its timed arm is
    the oracle port (OpenMP C restatement of the same arithmetic, O(Nk^2)),
    the stronger CPU line, and the reference's own Numba path is reported
    beside it (cpu_baseline_reference)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    wl = make_workload(a.workload, 0, a.nwires)
    threads = os.cpu_count() or 1
    vals = []
    for _ in range(max(1, a.warmup)):
        cpu_baseline(wl, 1.0, threads)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        vals.append(cpu_baseline(wl, min(a.cpu_seconds, 60.0 / max(1, a.steps)), threads))
    wall = time.perf_counter() - t0
    v = float(np.mean([x["value"] for x in vals]))
    cb = dict(vals[-1])
    cb["value"] = v
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": "wire*k*steps/s",
        "n_gpus": world,
        "steps": a.steps,
        "warmup": a.warmup,
        "ms_per_step": wall * 1e3 / a.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded configuration draws)",
        "config": config_for(a, wl, world),
        "form": "CPU oracle (OpenMP C restatement of the reference's path), all host threads",
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "wire*k*steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if not a.no_reference_baseline:
        try:
            line["cpu_baseline_reference"] = cpu_baseline_reference(wl, threads)
        except Exception as ex:
            line["cpu_baseline_reference"] = {"unavailable": f"{type(ex).__name__}: {ex}"}
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    if a.workload == "pstd":
        run_pstd(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
