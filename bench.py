#!/usr/bin/env python
"""Benchmark of the quantum-wire SBE step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c1] [--chunk S]

A bench step advances every wire of the workload by S time steps (one launch
of the fused step kernel per size class); the metric counts wire*k*steps,
i.e. sum_w Nk_w * S per bench step.  Default workload: configuration 1 (1024
wires, Nk ~ U[64,512] rounded to 32, RK4 with dt = 1 fs) in the batched
split form (exchange sums as exact int8-digit products on the tensor cores,
<= 1e-6 in P(t) against FP64); the plain FP64 form of the same workload is
timed in the same run and reported beside it ("plain").  --workload c4 runs
the continuous-batching server on the Poisson request stream of
configuration 4 and reports p50/p99 solve latency with the throughput.

Timing: W untimed bench steps, then K bench steps each bracketed by CUDA
events on the launching stream, with a 256 MiB write between them (L2 is
126 MB) outside the events; barrier + synchronize around the whole loop;
max over ranks.  `e2e` repeats the measurement through the public API with
each step's state copied in from pinned host memory and its P(t) + state
copied back inside the timed region (copies on their own streams,
overlapping the neighbouring steps' compute).  `--impl reference` times the CPU oracle (the
restatement of the reference's Numba path) on the host cores instead.
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
# DRAM bytes per state element and launch, from one ncu capture of each step
# kernel on a small configuration-3 case (dram__bytes_read.sum +
# dram__bytes_write.sum over 1184 x 256 elements; traffic grows with the
# elements a launch advances, not with its time steps)
DRAM_BYTES_PER_ELEMENT = {"split": 9.99e6 / (1184 * 256), "plain": 9.91e6 / (1184 * 256)}
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + write.sum of the step kernels on 1184 wires x "
                  "Nk 256, per element, times the elements of this step's launches")
METRIC = "SBE wire*k*steps/s at <=1e-6 rel err vs FP64 (batched vs plain); p50/p99 latency"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c1", choices=["c1", "c2", "c3", "c4"])
    ap.add_argument("--chunk", type=int, default=100, help="time steps per bench step")
    ap.add_argument("--form", default="split", choices=["plain", "split"],
                    help="split int8-digit tensor-core kernel or plain FP64 kernel")
    ap.add_argument("--no-plain", action="store_true",
                    help="skip the plain-form comparison of the split run")
    ap.add_argument("--rate", type=float, default=2000.0, help="c4: requests per second")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="c4: stream length")
    ap.add_argument("--capacity-requests", type=int, default=6000,
                    help="c4: requests of the saturated capacity run of each form")
    ap.add_argument("--nwires", type=int, default=0, help="override the workload's wire count")
    ap.add_argument("--acc-steps", type=int, default=3000,
                    help="split form: time steps of the accuracy check against the plain form "
                         "(the workload's duration, at most this; 0 skips it)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def make_workload(name, rank, nwires):
    from pulsesuite_b200 import workloads

    if name == "c4":
        # the request mix of the serving stream as a fixed batch of wires
        from pulsesuite_b200 import grid as pgrid
        from pulsesuite_b200 import abi, serve

        reqs = serve.poisson_stream(rate=2000.0, seconds=(nwires or 256) / 2000.0,
                                    seed=4 + 1000 * rank)
        grids = [pgrid.wire_grid(nk) for nk in serve.C4_NKS]
        w = np.concatenate([serve.wire_record(r, grids[serve.C4_NKS.index(r.nk)],
                                              table=serve.C4_NKS.index(r.nk)) for r in reqs])
        assert w.dtype == abi.WIRE_DTYPE
        return workloads.Workload(f"c4 request mix: {len(w)} wires", grids, w, 2500, 1e-15)
    kw = {"seed": 1 + 1000 * rank + {"c1": 0, "c2": 1, "c3": 2}[name]}
    if nwires:
        kw["nwires"] = nwires
    return workloads.CONFIGS[name](**kw)


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
# CPU baseline: the oracle (restatement of the reference's Numba path).
# ---------------------------------------------------------------------------
def cpu_baseline(wl, seconds, threads):
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
    if wl.screened and a.form == "split":
        a.form = "plain"  # the split form has no screened exchange
    S = a.chunk
    b = WireBatch(wl.grids, wl.wires, screened=wl.screened, p_cap=S, form=a.form)
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    units = wl.units_per_step * S
    flops_launch = wl.flops_per_step() * S

    def step(p_stride=1):
        b.rk4(S, wl.dt, p_stride=p_stride, stream=stream)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    # -- device-resident timing --------------------------------------------
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(a.steps)]
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        for i in range(a.steps):
            flush.fill_(float(i))
            evs[i][0].record(stream)
            b.rk4(S, wl.dt, p_stride=1, stream=stream)
            evs[i][1].record(stream)
        torch.cuda.synchronize()
    times = [e0.elapsed_time(e1) for e0, e1 in evs]
    total_ms = float(sum(times))
    if world > 1:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    value = units * a.steps * world / (total_ms * 1e-3)
    status = b.wires()["status"]
    plain = None
    if a.form == "split" and not a.no_plain:
        # the plain FP64 form of the same workload, same timing rules
        bp = WireBatch(wl.grids, wl.wires, screened=wl.screened, p_cap=S, form="plain")
        for _ in range(a.warmup):
            bp.rk4(S, wl.dt, stream=stream)
        pev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(a.steps)]
        torch.cuda.synchronize()
        for i in range(a.steps):
            flush.fill_(float(i))
            pev[i][0].record(stream)
            bp.rk4(S, wl.dt, p_stride=1, stream=stream)
            pev[i][1].record(stream)
        torch.cuda.synchronize()
        pms = float(sum(e0.elapsed_time(e1) for e0, e1 in pev))
        if world > 1:
            t = torch.tensor([pms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            pms = float(t.item())
        pval = units * a.steps * world / (pms * 1e-3)
        plain = {"value": pval, "ms_per_step": pms / a.steps, "split_over_plain": value / pval,
                 "gpu_launches": a.steps * bp.launches_per_call}
        del bp
    accuracy = None
    if a.form == "split" and not a.no_plain and a.acc_steps > 0:
        # the workload's own duration, bounded (at most ~1e10 wire*k*steps)
        # so the check stays a few seconds
        n_acc = min(wl.nsteps, a.acc_steps, max(50, int(1e10 // wl.units_per_step)))
        accuracy = split_accuracy(wl, n_acc, stream)

    # -- end to end through the public API: pinned host state in, P + state out.
    # Every step copies its input state from pinned host memory and reads its
    # P(t) records and final state back to pinned host memory; the copies run
    # on their own stream and overlap the neighbouring steps' compute, as a
    # caller streaming independent batches through the API would run them:
    #   upload stream:    H2D input(i+1) -> staging
    #   download stream:  D2H snapshot(i) -> host(i % 2)
    #   compute:      staging -> y, rk4, y/P -> snapshot(i % 2)
    # The timed region spans all K steps, from before the first upload to
    # after the last download.
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
    for i in range(a.steps):
        stream.wait_event(staged)
        flush.fill_(float(i))
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
        if i + 1 < a.steps:
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
    h2d = y_host.numel() * 8
    d2h = (P_out[0].numel() + y_out[0].numel()) * 8

    avg_launch_ms = total_ms / a.steps
    if a.form == "plain":
        peak = fp64_peak_tflops(torch, _lib, device)
        peak_source = "measured in this run: psb_probe_fp64_fma (FMA loop)"
        bound = "fp64"
    else:
        # the split algorithm's tensor-core work: 6 int8 digit products x 4
        # columns x Nk MACs (2 ops) per element and stage, 4 stages per step
        # (unpadded grid)
        flops_launch = float(np.sum(wl.nks.astype(np.float64) ** 2)) * 192.0 * S
        peak, peak_source = measured_bf16_peak()
        # dense int8 tensor rate is twice the bf16 rate on B200
        peak, peak_source = 2.0 * peak, "2 x " + peak_source
        bound = "tensor"
    achieved = flops_launch / (avg_launch_ms * 1e-3) / 1e12
    # DRAM bytes of one bench step's launches, scaled by elements from the
    # ncu captures of a small c3 case (split 9.99 MB, plain 9.91 MB for
    # 1184 x 256 elements: the FP64 state read once per launch)
    traffic = (DRAM_BYTES_PER_ELEMENT[a.form] * b.n_state) if b.n_state else None

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
        "dtype": "f64" if a.form == "plain" else "int8x3digits+s32acc+f64",
        "data": "synthetic (seeded configuration draws)",
        "config": {"workload": wl.name, "wires_per_gpu": len(wl.wires),
                   "wire_k_per_time_step": wl.units_per_step, "time_steps_per_bench_step": S,
                   "form": a.form, "l2": "256 MiB write between timed steps",
                   "parallelism": f"wires sharded, {world} independent GPU(s)"},
        "e2e": {"value": units * a.steps * world / (e2e_ms * 1e-3), "unit": "wire*k*steps/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"bound": bound, "achieved": achieved, "peak": peak, "unit": "TFLOP/s" if a.form == "plain" else "TOP/s",
                     "frac": achieved / peak, "traffic": traffic, "traffic_source": TRAFFIC_SOURCE,
                     "peak_source": peak_source, "flops_per_launch": flops_launch},
        "gpu_launches": a.steps * b.launches_per_call,
        "plain": plain,
        "accuracy": accuracy,
        "clocks": clk.summary(),
        "wire_status_ok": bool((status == 0).all()),
    }
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl, a.cpu_seconds, os.cpu_count() or 1)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    wl = make_workload(a.workload, 0, a.nwires)
    threads = os.cpu_count() or 1
    vals = []
    for _ in range(max(1, a.warmup)):
        cpu_baseline(wl, 1.0, threads)
    for _ in range(a.steps):
        vals.append(cpu_baseline(wl, min(a.cpu_seconds, 60.0 / max(1, a.steps)), threads))
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
        "ms_per_step": None,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded configuration draws)",
        "config": {"workload": wl.name, "form": "CPU oracle (restatement of the reference's "
                   "Numba path), all host threads"},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "wire*k*steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_serve(a):
    """Configuration 4: the continuous-batching server on the Poisson stream
    (split form), plus a saturated capacity run of both forms on the same
    request mix."""
    import torch

    from pulsesuite_b200 import serve

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    chunk = 50
    reqs = serve.poisson_stream(rate=a.rate, seconds=a.serve_seconds, seed=4 + 1000 * rank,
                                chunk=chunk)
    # warm-up: a few requests through each form
    warm = serve.poisson_stream(rate=200.0, seconds=0.1, seed=99, chunk=chunk)
    srv = serve.Server(form="split", chunk=chunk)
    srv.run(warm, realtime=False)
    with Clocks(local) as clk:
        res = srv.run(reqs, realtime=True)
    thr = srv.throughput()
    lat = srv.latency_percentiles((50, 99))
    ok = all(r.status == 0 for r in res)
    # saturated capacity of both forms on the same mix (all requests queued)
    cap = {}
    sat = serve.poisson_stream(rate=1e6, seconds=a.capacity_requests / 1e6, seed=5, chunk=chunk)
    # (one saturated run lasts about a second and varies by up to ~20 % from
    # run to run, so each form reports the median of three)
    cap_runs = {}
    for form in ("split", "plain"):
        vals = []
        for _ in range(3):
            s2 = serve.Server(form=form, chunk=chunk)
            s2.run(warm, realtime=False)
            s2.run(sat, realtime=False)
            vals.append(s2.throughput())
            del s2
            torch.cuda.synchronize()
        cap[form] = float(np.median(vals))
        cap_runs[form] = vals
    h2d = 136 * len(res)
    d2h = sum(16 * r.nsteps + 32 * r.nk for r in res)
    line = {
        "metric": METRIC,
        "value": thr,
        "unit": "wire*k*steps/s",
        "n_gpus": world,
        "steps": len(res),
        "warmup": len(warm),
        "ms_per_step": None,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int8x3digits+s32acc+f64",
        "data": "synthetic Poisson request stream (seeded)",
        "config": {"workload": f"c4: Poisson {a.rate:g}/s for {a.serve_seconds:g} s, Nk in "
                               "{64,128,256,512,1024} p={.3,.3,.2,.15,.05}, 1-4 ps at 1 fs, "
                               "150 GB HBM budget", "requests": len(res), "tick_steps": chunk,
                   "form": "split, continuous batching"},
        "latency_p50_s": lat.get(50),
        "latency_p99_s": lat.get(99),
        "capacity": {"split": cap["split"], "plain": cap["plain"],
                     "split_over_plain": cap["split"] / cap["plain"],
                     "requests": len(sat), "runs": cap_runs, "statistic": "median of 3"},
        "e2e": {"value": thr, "unit": "wire*k*steps/s", "h2d_bytes_per_step": h2d / max(1, len(res)),
                "d2h_bytes_per_step": d2h / max(1, len(res))},
        "roofline": None,
        "gpu_launches": None,
        "clocks": clk.summary(),
        "wire_status_ok": ok,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "c4":
        run_serve(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
