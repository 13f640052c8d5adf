"""Continuous-batching SBE solve server (serving configuration c4).

Requests are single-wire SBE solves (own Nk, pulse, dephasing and
duration) arriving over time.  The server keeps every admitted solve's state
resident on the device in a slot pool, and each tick advances all resident
solves by ``chunk`` RK4 steps with one launch per size class of the fused
step kernel (split int8-digit tensor-core form or plain FP64 form).
Between ticks it retires finished solves (their P(t) records and final
state are copied to pinned host memory asynchronously) and admits waiting
requests as slots and the HBM budget free up, so new work joins the
running batch without waiting for the batch to drain.

    srv = Server(form="split")
    results = srv.run(stream_of_requests)      # list of Result
    srv.latency_percentiles()                  # p50 / p99 seconds

A result does not depend on which other solves share its launches: wires
are independent in both step kernels (each CTA's arithmetic for a wire
reads only that wire's state, its own pulse and the shared Coulomb table),
so a solve returns the same numbers alone and in any mix.

Host-side logic (request stream, slot allocation, HBM accounting) is plain
Python and tested without a GPU; the device path needs the sm_100a library.
"""

import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi

EV = 1.602176634e-19
# Nk classes of the serving stream and their probabilities
C4_NKS = (64, 128, 256, 512, 1024)
C4_PROBS = (0.3, 0.3, 0.2, 0.15, 0.05)

# Cost model of the split-form scheduler: time of one CTA for one 50-step
# launch (ms, one CTA per SM, full waves), measured on a B200, by grid size
# and wires per CTA.  8 wires double the width of every MMA at the same
# issue count, so a CTA of 8 takes only 1.2-1.6x as long as a CTA of 4:
# more throughput, more latency.  Other grid sizes scale from the nearest
# entry by Nk^2 (the exchange work per wire).
SPLIT_CTA_MS = {(64, 4): 0.49, (64, 8): 0.73, (128, 4): 0.58, (128, 8): 0.84,
                (256, 4): 0.90, (256, 8): 1.37, (512, 4): 2.53, (512, 8): 3.96,
                (1024, 4): 8.15, (1024, 8): 9.71}


def split_cta_cost(nk, w):
    ref = min((k for k, ww in SPLIT_CTA_MS if ww == w), key=lambda k: abs(math.log(k / nk)))
    return SPLIT_CTA_MS[(ref, w)] * (nk / ref) ** 2


def choose_wires_per_cta(counts, sms, w8_ok=lambda nk: True):
    """Wires per CTA (4 or 8) of each grid size for one tick.

    counts: {nk: solves of that size in the tick}.  A tick lasts about
    max(longest CTA, total CTA time / SMs): with few solves the longest CTA
    sets it and 4 wires per CTA give the shorter tick (lower latency); once
    the SMs are full the total sets it and 8 wires per CTA give more
    throughput.  Starting from 4 everywhere, each size (largest first)
    moves to 8 if that shortens the estimated tick, or keeps it and frees
    SM time."""
    w = {nk: 4 for nk, c in counts.items() if c}

    def tick(wm):
        total = sum(-(-counts[nk] // wm[nk]) * split_cta_cost(nk, wm[nk]) for nk in wm)
        return (max(max(split_cta_cost(nk, wm[nk]) for nk in wm), total / sms), total)

    if not w:
        return w
    best = tick(w)
    for nk in sorted(w, reverse=True):
        if not w8_ok(nk):
            continue
        trial = dict(w)
        trial[nk] = 8
        t = tick(trial)
        if t < best:
            w, best = trial, t
    return w


@dataclass
class SolveRequest:
    rid: int
    arrival: float  # seconds after the start of the stream
    nk: int
    theta: float  # pulse area
    det_eV: float  # detuning
    fwhm: float
    T2: float
    nsteps: int
    dt: float = 1e-15


@dataclass
class Result:
    rid: int
    nk: int
    nsteps: int
    arrival: float
    admitted: float
    finished: float
    status: int
    P: np.ndarray = field(repr=False)  # complex (nsteps,)
    y: np.ndarray = field(repr=False)  # (nk, 4) float64

    @property
    def latency(self):
        return self.finished - self.arrival


def poisson_stream(rate=2000.0, seconds=60.0, seed=4, chunk=50, nks=C4_NKS, probs=C4_PROBS,
                   dur_ps=(1.0, 4.0), dt=1e-15):
    """Configuration-4 request stream: Poisson arrivals at ``rate``/s for
    ``seconds``; Nk from ``nks`` with ``probs``; duration U[1, 4] ps at dt
    (rounded up to whole ticks of ``chunk`` steps); pulse area, detuning,
    FWHM and T2 as configuration 1."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    rid = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= seconds:
            break
        nk = int(rng.choice(nks, p=probs))
        steps = int(round(rng.uniform(*dur_ps) * 1e-12 / dt))
        steps = max(chunk, int(math.ceil(steps / chunk)) * chunk)
        out.append(SolveRequest(rid, t, nk, float(rng.uniform(0.1 * np.pi, 2 * np.pi)),
                                float(rng.uniform(-50e-3, 50e-3)),
                                float(rng.uniform(20e-15, 200e-15)),
                                float(rng.uniform(50e-15, 300e-15)), steps, dt))
        rid += 1
    return out


def request_bytes(nk, nsteps, form):
    """Resident device bytes of one solve: FP64 state, the split form's
    workspace and its P(t) records."""
    ws = 64 * nk if form == "split" else 0
    return 32 * nk + ws + 16 * nsteps


class SlotPool:
    """Free-slot bookkeeping per Nk class plus an HBM budget (host only)."""

    def __init__(self, capacity, budget_bytes):
        self.capacity = dict(capacity)
        self.free = {nk: list(range(c - 1, -1, -1)) for nk, c in self.capacity.items()}
        self.budget = float(budget_bytes)
        self.used = 0.0

    def try_take(self, nk, nbytes):
        if nk not in self.free or not self.free[nk] or self.used + nbytes > self.budget:
            return None
        self.used += nbytes
        return self.free[nk].pop()

    def give_back(self, nk, slot, nbytes):
        self.free[nk].append(slot)
        self.used -= nbytes

    def in_use(self, nk):
        return self.capacity[nk] - len(self.free[nk])


def default_capacity(nks=C4_NKS):
    """Slots per Nk class (concurrent solves); the HBM budget admits within
    these."""
    return {nk: max(256, int(4096 * 256 // max(nk, 256))) for nk in nks}


class Server:
    """Device slot pool + tick loop (see module docstring)."""

    def __init__(self, form="split", chunk=50, max_steps=4000, capacity=None,
                 hbm_budget=150e9, nks=C4_NKS):
        import torch
        from scipy.constants import hbar

        from . import _lib, coulomb, device
        from . import grid as pgrid

        device.require_cuda()
        if form not in ("split", "plain"):
            raise ValueError("form must be 'split' or 'plain'")
        self.torch, self._lib, self.device = torch, _lib, device
        self.form, self.chunk, self.max_steps = form, int(chunk), int(max_steps)
        if self.max_steps % self.chunk:
            raise ValueError("max_steps must be a multiple of chunk")
        self.nks = tuple(int(n) for n in nks)
        self.grids = [pgrid.wire_grid(nk) for nk in self.nks]
        tables, self.tabdata = coulomb.grid_tables(self.grids)
        self.h_tables = np.ascontiguousarray(tables)
        self.d_tables = device.to_device(self.h_tables)
        cap = dict(capacity or default_capacity(self.nks))
        self.pool = SlotPool(cap, hbm_budget)
        # slot layout: class c holds cap[nk] slots; global slot index g
        self.cls_base, base, off = {}, 0, 0
        self.slot_off = []
        for ti, nk in enumerate(self.nks):
            self.cls_base[nk] = base
            for s in range(cap[nk]):
                self.slot_off.append(off + s * nk)
            base += cap[nk]
            off += cap[nk] * nk
        self.nslots = base
        self.n_state = off
        w = np.zeros(self.nslots, dtype=abi.WIRE_DTYPE)
        for ti, nk in enumerate(self.nks):
            b = self.cls_base[nk]
            w["table"][b:b + cap[nk]] = ti
        w["off"] = np.asarray(self.slot_off, dtype=np.int64)
        w["p_off"] = np.arange(self.nslots, dtype=np.int64) * self.max_steps
        self.h_wires = w
        self.d_wires = device.to_device(w)
        self._wires_i64 = self.d_wires.view(torch.int64).view(self.nslots, abi.WIRE_DTYPE.itemsize // 8)
        self._p_off_col = abi.WIRE_DTYPE.fields["p_off"][1] // 8
        self.y = torch.zeros((self.n_state, 4), dtype=torch.float64, device="cuda")
        self.P = torch.zeros((self.nslots * self.max_steps, 2), dtype=torch.float64, device="cuda")
        lib = _lib.load()
        if form == "split":
            self.ws = torch.empty(int(lib.psb_split_ws_bytes(self.n_state)), dtype=torch.uint8,
                                  device="cuda")
            # wires per CTA are chosen per tick (choose_wires_per_cta); 8
            # only where that group fits in shared memory
            self.w8_max = int(lib.psb_split_max_nk(8))
            self.sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        self.model = abi.model_array(hbar)
        self.streams = [torch.cuda.Stream() for _ in self.nks]
        self.copy_stream = torch.cuda.Stream()
        self.isz = abi.WIRE_DTYPE.itemsize
        self._wires_rows = self.d_wires.view(self.nslots, self.isz)
        # per-tick metadata goes through a ring of pinned staging buffers and
        # one asynchronous copy per tick (the ring depth exceeds the number
        # of ticks allowed in flight, so a buffer is never rewritten while
        # its copy may still be pending)
        self.ring = 3
        nb = max(1 << 20, 64 * self.nslots + 8 * self.nslots * abi.SPLIT_GROUP_DTYPE.itemsize)
        self.stage_h = [torch.empty(nb, dtype=torch.uint8, pin_memory=True) for _ in range(self.ring)]
        self.stage_d = [torch.empty(nb, dtype=torch.uint8, device="cuda") for _ in range(self.ring)]
        self.tick = 0
        self.active = {}  # global slot -> [request, steps_done, admitted_time, nbytes]
        self.pending = []  # retiring batches: (event, entries, host buffers)
        self.results = []

    # -- staging -------------------------------------------------------------------
    class _Stage:
        """Packs numpy arrays into a pinned buffer; after ``push`` their
        device copies are views of the device buffer at the same offsets."""

        def __init__(self, h, d):
            self.h, self.d, self.n, self.items = h, d, 0, []

        def add(self, arr):
            arr = np.ascontiguousarray(arr)
            raw = arr.view(np.uint8).reshape(-1)
            o = (self.n + 15) & ~15
            if o + raw.size > self.h.numel():
                raise RuntimeError("serving stage buffer too small")
            self.h.numpy()[o:o + raw.size] = raw
            self.n = o + raw.size
            return (o, raw.size)

        def view(self, ref, dtype):
            o, n = ref
            return self.d[o:o + n].view(dtype)

    def _stage(self):
        i = self.tick % self.ring
        return Server._Stage(self.stage_h[i], self.stage_d[i])

    def _push(self, st):
        if st.n:
            self.stage_d[self.tick % self.ring][:st.n].copy_(
                self.stage_h[self.tick % self.ring][:st.n], non_blocking=True)

    def _rows(self, offs, nks, total):
        """Device row indices of the state ranges [off, off + nk) (total =
        sum of nk, known on the host, so nothing synchronises)."""
        torch = self.torch
        starts = torch.repeat_interleave(offs, nks, output_size=total)
        base = torch.repeat_interleave(torch.cumsum(nks, 0) - nks, nks, output_size=total)
        return starts + (torch.arange(total, device="cuda") - base)

    # -- admission / launch / retirement ---------------------------------------------
    def _admit_batch(self, reqs, now, st):
        """Admit as many of ``reqs`` as slots and budget allow; returns the
        ones left waiting.  Their wire descriptors and zeroed state reach the
        device with this tick's staged copy."""
        recs, slots, left = [], [], []
        for req in reqs:
            if req.nsteps > self.max_steps:
                raise ValueError(f"request {req.rid}: {req.nsteps} steps > max_steps")
            nbytes = request_bytes(req.nk, req.nsteps, self.form)
            s = self.pool.try_take(req.nk, nbytes)
            if s is None:
                left.append(req)
                continue
            g = self.cls_base[req.nk] + s
            ti = self.nks.index(req.nk)
            rec = wire_record(req, self.grids[ti], table=ti, off=self.slot_off[g],
                              p_off=g * self.max_steps)
            self.h_wires[g] = rec[0]
            recs.append(rec)
            slots.append(g)
            self.active[g] = [req, 0, now, nbytes]
        if slots:
            sl = np.asarray(slots, dtype=np.int64)
            nk_adm = np.asarray([self.active[g][0].nk for g in slots], dtype=np.int64)
            self._adm = (st.add(np.concatenate(recs)), st.add(sl),
                         st.add(np.asarray([self.slot_off[g] for g in slots], dtype=np.int64)),
                         st.add(nk_adm), len(slots), int(nk_adm.sum()))
        else:
            self._adm = None
        return left

    def _apply_admissions(self, st):
        if self._adm is None:
            return
        torch = self.torch
        r_rec, r_sl, r_off, r_nk, k, total = self._adm
        idx = st.view(r_sl, torch.int64)
        self._wires_rows[idx] = st.view(r_rec, torch.uint8).view(k, self.isz)
        rows = self._rows(st.view(r_off, torch.int64), st.view(r_nk, torch.int64), total)
        self.y.index_fill_(0, rows, 0.0)

    def _launch(self, st):
        torch = self.torch
        if not self.active:
            return
        slots = np.fromiter(self.active.keys(), dtype=np.int64)
        done = np.array([self.active[g][1] for g in slots], dtype=np.int64)
        r_idx = st.add(slots)
        r_val = st.add(slots * self.max_steps + done)  # P(t) records append
        # solves that finish with this tick: their slots and state ranges
        fin = slots[done + self.chunk >= np.array([self.active[g][0].nsteps for g in slots])]
        if fin.size:
            self._fin = (fin, st.add(fin),
                         st.add(np.asarray([self.slot_off[g] for g in fin], dtype=np.int64)),
                         st.add(np.asarray([self.active[g][0].nk for g in fin], dtype=np.int64)))
        else:
            self._fin = None
        tables = self.h_wires["table"][slots]
        if self.form == "split":
            counts = {nk: int((tables == ti).sum()) for ti, nk in enumerate(self.nks)}
            self.wg = choose_wires_per_cta(counts, self.sms, lambda nk: nk <= self.w8_max)
        plan = []
        # largest grids first: their CTAs run longest, so they start before
        # the short ones fill the SMs
        for ti, nk in sorted(enumerate(self.nks), key=lambda t: -t[1]):
            sel = slots[tables == ti]
            if sel.size == 0:
                continue
            if self.form == "split":
                wg = self.wg[nk]
                ng = (sel.size + wg - 1) // wg
                grp = np.zeros(ng, dtype=abi.SPLIT_GROUP_DTYPE)
                grp["table"] = ti
                grp["wire"] = -1
                padded = np.full(ng * wg, -1, dtype=np.int32)
                padded[:sel.size] = sel
                grp["wire"][:, :wg] = padded.reshape(ng, wg)
                grp["nw"] = wg
                grp["nw"][-1] = sel.size - (ng - 1) * wg
                plan.append((ti, nk, st.add(grp), ng, wg))
            else:
                plan.append((ti, nk, st.add(sel.astype(np.int32)), sel.size, 0))
        self._push(st)
        self._apply_admissions(st)
        self._wires_i64[st.view(r_idx, torch.int64), self._p_off_col] = st.view(r_val, torch.int64)
        main = torch.cuda.current_stream()
        fork = torch.cuda.Event()
        fork.record(main)
        joins = []
        common = (self.device.ptr(self.d_tables), len(self.h_tables), self.device.ptr(self.tabdata),
                  self.tabdata.numel(), self.device.ptr(self.d_wires), self.nslots)
        dt = float(next(iter(self.active.values()))[0].dt)
        for ti, nk, ref, n, wg in plan:
            sm = self.streams[ti]
            sm.wait_event(fork)
            ptr = self.device.ptr(st.view(ref, torch.uint8))
            if self.form == "split":
                self._lib.call("psb_rk4_split", *common, ptr, n, wg, nk, self.device.ptr(self.y),
                               self.n_state, self.device.ptr(self.ws), self.ws.numel(), self.chunk,
                               dt, self.device.ptr(self.P), self.P.shape[0], 1, self.max_steps,
                               abi.as_ptr(self.model), self.device.stream_ptr(sm))
            else:
                flags = abi.PSB_TAB_SHARED_V if (self.h_tables["flags"][ti] & abi.PSB_TAB_SHARED_V) else 0
                self._lib.call("psb_rk4_f64", *common, ptr, n, self.device.ptr(self.y), self.n_state,
                               nk, flags, self.chunk, dt, self.device.ptr(self.P), self.P.shape[0],
                               1, self.max_steps, abi.as_ptr(self.model), self.device.stream_ptr(sm))
            ev = torch.cuda.Event()
            ev.record(sm)
            joins.append(ev)
        for ev in joins:
            main.wait_event(ev)
        for g in slots:
            self.active[int(g)][1] += self.chunk

    def _retire(self, st):
        torch = self.torch
        if getattr(self, "_fin", None) is None:
            return
        fin, r_fin, r_off, r_nk = self._fin
        self._fin = None
        entries = [(int(g), *self.active.pop(int(g))) for g in fin]
        nks = np.asarray([e[1].nk for e in entries], dtype=np.int64)
        fin_t = st.view(r_fin, torch.int64)
        main = torch.cuda.current_stream()
        rows = self._rows(st.view(r_off, torch.int64), st.view(r_nk, torch.int64), int(nks.sum()))
        # gather on the main stream (ordered after this tick's launches) ...
        Pg = self.P.view(self.nslots, self.max_steps, 2).index_select(0, fin_t)
        yg = self.y.index_select(0, rows)
        wg = self._wires_rows.index_select(0, fin_t)
        ev0 = torch.cuda.Event()
        ev0.record(main)
        cs = self.copy_stream
        cs.wait_event(ev0)
        # ... and copy to pinned host memory on the copy stream
        with torch.cuda.stream(cs):
            hP = torch.empty(Pg.shape, dtype=torch.float64, pin_memory=True)
            hy = torch.empty(yg.shape, dtype=torch.float64, pin_memory=True)
            hw = torch.empty(wg.shape, dtype=torch.uint8, pin_memory=True)
            hP.copy_(Pg, non_blocking=True)
            hy.copy_(yg, non_blocking=True)
            hw.copy_(wg, non_blocking=True)
            Pg.record_stream(cs)
            yg.record_stream(cs)
            wg.record_stream(cs)
            ev = torch.cuda.Event()
            ev.record(cs)
        self.pending.append((ev, entries, nks, hP, hy, hw))

    def _collect(self, block=False):
        keep = []
        for item in self.pending:
            ev, entries, nks, hP, hy, hw = item
            if block:
                ev.synchronize()
            elif not ev.query():
                keep.append(item)
                continue
            now = time.perf_counter() - self.t_start
            P, Y = hP.numpy(), hy.numpy()
            W = hw.numpy().reshape(-1).view(abi.WIRE_DTYPE)
            o = 0
            for i, (g, req, _, admitted, nbytes) in enumerate(entries):
                p = P[i, :req.nsteps]
                self.results.append(Result(req.rid, req.nk, req.nsteps, req.arrival, admitted, now,
                                           int(W["status"][i]), p[:, 0] + 1j * p[:, 1],
                                           Y[o:o + req.nk].copy()))
                o += req.nk
                self.pool.give_back(req.nk, g - self.cls_base[req.nk], nbytes)
        self.pending = keep

    def run(self, requests, realtime=True, max_inflight_ticks=2):
        """Serve ``requests``.  realtime: arrivals are honoured on the wall
        clock (the Poisson stream), else every request is available from the
        start (throughput / capacity runs)."""
        torch = self.torch
        assert max_inflight_ticks < self.ring
        queue = sorted(requests, key=lambda r: r.arrival)
        qi, n = 0, len(queue)
        waiting = []
        self.results = []
        self.t_start = time.perf_counter()
        tick_events = []
        while len(self.results) < n:
            now = time.perf_counter() - self.t_start
            while qi < n and (not realtime or queue[qi].arrival <= now):
                waiting.append(queue[qi])
                qi += 1
            self._collect()
            st = self._stage()
            waiting = self._admit_batch(waiting, now, st)
            if self.active:
                self._launch(st)
                self._retire(st)
                ev = torch.cuda.Event()
                ev.record(torch.cuda.current_stream())
                tick_events.append(ev)
                self.tick += 1
                while len(tick_events) > max_inflight_ticks:
                    tick_events.pop(0).synchronize()
            elif self.pending:
                self._collect(block=True)
            elif qi < n and realtime:
                time.sleep(max(0.0, min(1e-3, queue[qi].arrival - now)))
        torch.cuda.synchronize()
        self._collect(block=True)
        self.elapsed = time.perf_counter() - self.t_start
        return sorted(self.results, key=lambda r: r.rid)

    def latency_percentiles(self, qs=(50, 99)):
        lat = np.array([r.latency for r in self.results])
        return {q: float(np.percentile(lat, q)) for q in qs} if lat.size else {}

    def throughput(self):
        """Completed wire*k*steps per second of the run."""
        work = sum(r.nk * r.nsteps for r in self.results)
        return work / self.elapsed if self.elapsed > 0 else 0.0


def wire_record(req, grid, table=0, off=0, p_off=0):
    """Wire descriptor of a solve request (zero initial time and status):
    rotating-frame gap = -detuning, dephasing rate 1/T2, Gaussian pulse of
    area theta centred at 3 FWHM (configuration-1 conventions)."""
    from .grid import gaussian_amplitude

    rec = np.zeros(1, dtype=abi.WIRE_DTYPE)
    mscale = grid.ehint * grid.dcv / 2.0
    rec["table"] = table
    rec["npulse"] = 1
    rec["off"] = off
    rec["gap"] = -req.det_eV * EV
    rec["gamma"] = 1.0 / req.T2
    rec["mscale"] = mscale
    rec["pscale"] = grid.pscale
    rec["amp"][0, 0] = gaussian_amplitude(req.theta, req.fwhm, mscale)
    rec["t0"][0, 0] = 3.0 * req.fwhm
    rec["fwhm"][0, :] = req.fwhm
    rec["p_off"] = p_off
    return rec
