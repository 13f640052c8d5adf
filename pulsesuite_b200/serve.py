"""Continuous-batching SBE solve server (serving configuration c4).

Requests are single-wire SBE solves (own Nk, pulse, dephasing and
duration) arriving over time.  The server keeps every admitted solve's state
resident on the device in a slot pool.  Each size class (Nk) is a lane
with its own CUDA stream: a tick of a lane advances all of that class's
resident solves by ``chunk`` RK4 steps with one launch of the fused step
kernel (split int8-digit tensor-core form or plain FP64 form), retires the
solves that finish (their P(t) records and final state are copied to
pinned host memory asynchronously) and admits waiting requests of the class
as slots and the HBM budget free up, so new work joins the running batch
without waiting for it to drain.  The lanes tick independently and their
launches run concurrently, so a small solve is not held to the pace of the
largest grid.

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

import collections
import functools
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import abi

EV = 1.602176634e-19
# Result.status of a request cancelled before it finished (host-side status;
# the kernel statuses are the PSB_* codes, all >= -6)
STATUS_CANCELLED = -100
# Nk classes of the serving stream and their probabilities
C4_NKS = (64, 128, 256, 512, 1024)
C4_PROBS = (0.3, 0.3, 0.2, 0.15, 0.05)

# Default cost model of the split-form scheduler (the server measures its
# own with tune.SplitTuner on the device it runs on): time of one CTA for
# one 50-step launch (ms, one CTA per SM, full waves), measured on a B200,
# by grid size and wires per CTA.  8 wires double the width of every MMA at
# the same issue count, so a CTA of 8 takes only 1.2-1.6x as long as a CTA
# of 4: more throughput, more latency.  Other grid sizes scale from the
# nearest entry by Nk^2 (the exchange work per wire).
SPLIT_CTA_MS = {(64, 4): 0.49, (64, 8): 0.73, (128, 4): 0.58, (128, 8): 0.84,
                (256, 4): 0.90, (256, 8): 1.37, (512, 4): 2.53, (512, 8): 3.96,
                (1024, 4): 8.15, (1024, 8): 9.71}


@functools.lru_cache(maxsize=None)
def split_cta_cost(nk, w):
    ref = min((k for k, ww in SPLIT_CTA_MS if ww == w), key=lambda k: abs(math.log(k / nk)))
    return SPLIT_CTA_MS[(ref, w)] * (nk / ref) ** 2


def choose_wires_per_cta(counts, sms, w8_ok=lambda nk: True, cost=None, allowed=None):
    """Wires per CTA of each grid size for one tick.

    counts: {nk: solves of that size in the tick}.  A tick lasts about
    max(longest CTA, total CTA time / SMs): with few solves the longest CTA
    sets it and narrow groups give the shorter tick (lower latency); once
    the SMs are full the total sets it and wide groups give more
    throughput.  Starting from the narrowest group everywhere, each size
    (largest first) widens if that shortens the estimated tick, or keeps it
    and frees SM time (tune.choose_widths).  Without ``cost`` / ``allowed``
    the default table above is used with widths 4 and 8 (8 where w8_ok)."""
    from .tune import choose_widths

    if cost is None:
        cost = split_cta_cost
    if allowed is None:
        def allowed(nk):
            return (4, 8) if w8_ok(nk) else (4,)
    return choose_widths(counts, sms, cost, allowed)


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
    """Device slot pool + tick loop (see module docstring).

    max_inflight_ticks: ticks a lane may have queued on its stream before
    the host waits for the oldest (2: lower latency; 3 measured the same
    saturated capacity within the run-to-run spread)."""

    def __init__(self, form="split", chunk=50, max_steps=4000, capacity=None,
                 hbm_budget=150e9, nks=C4_NKS, max_inflight_ticks=2, hbm_headroom=2 << 30):
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
        # The resident pool (every slot's state, workspace and P(t) records)
        # is allocated once, here, and sized by the device's free memory
        # now: if it does not fit min(hbm_budget, free - headroom), every
        # class is scaled down (at least one slot each).  Requests are then
        # admitted into free slots within the same byte budget.
        free, total = torch.cuda.mem_get_info()
        self.hbm_free_at_start, self.hbm_total = int(free), int(total)
        per_slot = {nk: request_bytes(nk, self.max_steps, form) for nk in self.nks}
        need = sum(cap[nk] * per_slot[nk] for nk in self.nks)
        fit = min(float(hbm_budget), float(free) - float(hbm_headroom))
        if need > fit:
            scale = max(0.0, fit) / need
            cap = {nk: max(1, int(cap[nk] * scale)) for nk in self.nks}
            need = sum(cap[nk] * per_slot[nk] for nk in self.nks)
        self.pool_bytes = need
        self.pool = SlotPool(cap, min(float(hbm_budget), float(need)))
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
        self.slot_off_arr = np.asarray(self.slot_off, dtype=np.int64)
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
            # wires per CTA are chosen per tick (choose_wires_per_cta) from
            # per-CTA costs measured on this device for the served grids
            from .tune import shared_tuner

            self.tuner = shared_tuner()
            self.tuner.table(self.nks)
            self.sms = self.tuner.sms
            # per-tick cost of a CTA: the tuner's per-step cost times the tick
            self._cta_cost = functools.lru_cache(maxsize=None)(
                lambda nk, w: self.tuner.cost(nk, w) * self.chunk)
        self.model = abi.model_array(hbar)
        self.copy_stream = torch.cuda.Stream()
        self.isz = abi.WIRE_DTYPE.itemsize
        self._wires_rows = self.d_wires.view(self.nslots, self.isz)
        # one lane per size class: its own stream, its own ticks, its own
        # queue and pinned staging ring (per-tick metadata goes through one
        # asynchronous copy; the ring is deeper than the ticks allowed in
        # flight, so a buffer is never rewritten while its copy may pend).
        #
        # The lanes' streams get priorities by grid size, the largest grid
        # highest: its CTAs run longest and set the tail (and the p99), so
        # when SMs free up the CTA scheduler gives them to it first.
        self.max_inflight = int(max_inflight_ticks)  # queued ticks per lane
        self.ring = self.max_inflight + 1
        self.lanes = []
        least, greatest = torch.cuda.Stream.priority_range()
        rank = {nk: r for r, nk in enumerate(sorted(self.nks, reverse=True))}
        for ti, nk in enumerate(self.nks):
            nb = max(1 << 16, 64 * cap[nk] + 8 * cap[nk] * abi.SPLIT_GROUP_DTYPE.itemsize)
            prio = min(least, greatest + rank[nk])
            self.lanes.append(Server._Lane(
                ti, nk, self.cls_base[nk], cap[nk], torch.cuda.Stream(priority=prio),
                [torch.empty(nb, dtype=torch.uint8, pin_memory=True) for _ in range(self.ring)],
                [torch.empty(nb, dtype=torch.uint8, device="cuda") for _ in range(self.ring)]))
        self.tick = 0     # lane ticks issued, all lanes
        self.active = {}  # global slot -> [request, steps_done, admitted_time, nbytes]
        self.steps_done = np.zeros(self.nslots, dtype=np.int64)  # per slot, of its solve
        self.steps_req = np.zeros(self.nslots, dtype=np.int64)
        self._ar = {nk: torch.arange(nk, dtype=torch.int64, device="cuda") for nk in self.nks}
        self.pending = []  # retiring batches: (event, entries, host views, pinned buffer)
        self._pin_free = []  # pinned host buffers whose contents were collected
        self.results = []
        # launch arguments that do not change between ticks
        self._common = (device.ptr(self.d_tables), len(self.h_tables), device.ptr(self.tabdata),
                        self.tabdata.numel(), device.ptr(self.d_wires), self.nslots)
        self._y_ptr, self._P_ptr = device.ptr(self.y), device.ptr(self.P)
        self._model_ptr = abi.as_ptr(self.model)
        self._ws_ptr = device.ptr(self.ws) if form == "split" else None
        self._cancel = set()  # request ids to cancel
        self._cancelled = set()  # active slots cancelled (retire with STATUS_CANCELLED)
        self.reset_counters()

    def reset_counters(self):
        """Zero the host<->device byte counters and the tick count (bytes of
        the tensors each tick copies: staged metadata in, records and states
        out)."""
        self.h2d_bytes = 0
        self.d2h_bytes = 0
        self.tick_count = 0

    class _Lane:
        """One size class: stream, tick count, waiting requests, active
        slots, events of its ticks in flight, staging ring."""

        def __init__(self, ti, nk, base, cap, stream, stage_h, stage_d):
            self.ti, self.nk, self.stream = ti, nk, stream
            self.stage_h, self.stage_d = stage_h, stage_d
            self.tick = 0
            self.waiting = collections.deque()
            # active slots of the class as a mask over its slot range (the
            # sorted slot list of a tick is one flatnonzero)
            self.base = base
            self.mask = np.zeros(cap, dtype=bool)
            self.nactive = 0
            self.inflight = []

        @property
        def slots(self):
            return self.nactive > 0

        def slot_array(self):
            return self.base + np.flatnonzero(self.mask).astype(np.int64)

    # -- staging -------------------------------------------------------------------
    class _Stage:
        """Packs numpy arrays into a pinned buffer; after ``push`` their
        device copies are views of the device buffer at the same offsets."""

        def __init__(self, h, d):
            self.h, self.d, self.n = h, d, 0

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

        def push(self):
            """Copy to the device on the current stream."""
            if self.n:
                self.d[:self.n].copy_(self.h[:self.n], non_blocking=True)

    def _rows(self, offs, nk):
        """Device row indices of the state ranges [off, off + nk) of one
        size class, as one broadcast add (nothing synchronises)."""
        return (offs.view(-1, 1) + self._ar[nk].view(1, -1)).view(-1)

    # -- one tick of one lane ------------------------------------------------------------
    def _admit(self, lane, now, st):
        """Admit as many of the lane's waiting requests as slots and budget
        allow; returns the staged admission or None.  Their wire descriptors
        and zeroed state reach the device with this tick's staged copy."""
        reqs, slots = [], []
        while lane.waiting:
            req = lane.waiting[0]
            nbytes = request_bytes(req.nk, req.nsteps, self.form)
            sl = self.pool.try_take(req.nk, nbytes)
            if sl is None:
                break  # the class's slots or the byte budget are used up
            lane.waiting.popleft()
            g = self.cls_base[req.nk] + sl
            reqs.append(req)
            slots.append(g)
            self.active[g] = [req, 0, now, nbytes]
            lane.mask[sl] = True
        if not slots:
            return None
        # the descriptors of every admitted solve in one pass (the same
        # values wire_record gives one request)
        g = np.asarray(slots, dtype=np.int64)
        offs = self.slot_off_arr[g]
        recs = wire_records(reqs, self.grids[lane.ti], table=lane.ti, offs=offs,
                            p_offs=g * self.max_steps)
        self.h_wires[g] = recs
        self.steps_done[g] = 0
        self.steps_req[g] = [r.nsteps for r in reqs]
        lane.nactive += len(slots)
        return st.add(recs), st.add(g), st.add(offs), len(slots)

    def _tick(self, lane, now):
        """Admit, advance and retire one size class by ``chunk`` steps, all
        on the lane's stream.  Returns False when the lane has nothing to do."""
        torch = self.torch
        i = lane.tick % self.ring
        st = Server._Stage(lane.stage_h[i], lane.stage_d[i])
        adm = self._admit(lane, now, st)
        if not lane.slots:
            return False
        slots = lane.slot_array()
        done = self.steps_done[slots]
        r_idx = st.add(slots)
        r_val = st.add(slots * self.max_steps + done)  # P(t) records append
        # solves that finish with this tick
        fin = slots[done + self.chunk >= self.steps_req[slots]]
        r_fin = r_foff = None
        if fin.size:
            r_fin = st.add(fin)
            r_foff = st.add(self.slot_off_arr[fin])
        nk, ti = lane.nk, lane.ti
        if self.form == "split":
            # the classes share the SMs, so the choice sees every lane's load
            counts = {ln.nk: ln.nactive for ln in self.lanes}
            wg = choose_wires_per_cta(counts, self.sms, cost=self._cta_cost,
                                      allowed=self.tuner.allowed)[nk]
            ng = (slots.size + wg - 1) // wg
            grp = np.zeros(ng, dtype=abi.SPLIT_GROUP_DTYPE)
            grp["table"] = ti
            grp["wire"] = -1
            padded = np.full(ng * wg, -1, dtype=np.int32)
            padded[:slots.size] = slots
            grp["wire"][:, :wg] = padded.reshape(ng, wg)
            grp["nw"] = wg
            grp["nw"][-1] = slots.size - (ng - 1) * wg
            r_grp, n_launch = st.add(grp), ng
        else:
            wg = 0
            r_grp, n_launch = st.add(slots.astype(np.int32)), slots.size
        common = self._common
        dt = float(self.active[int(slots[0])][0].dt)
        sm = lane.stream
        self.h2d_bytes += st.n
        self.tick_count += 1
        with torch.cuda.stream(sm):
            st.push()
            if adm is not None:
                r_rec, r_sl, r_off, k = adm
                idx = st.view(r_sl, torch.int64)
                self._wires_rows[idx] = st.view(r_rec, torch.uint8).view(k, self.isz)
                self.y.index_fill_(0, self._rows(st.view(r_off, torch.int64), nk), 0.0)
            self._wires_i64[st.view(r_idx, torch.int64), self._p_off_col] = st.view(r_val, torch.int64)
            ptr = self.device.ptr(st.view(r_grp, torch.uint8))
            if self.form == "split":
                self._lib.call("psb_rk4_split", *common, ptr, n_launch, wg, nk,
                               self._y_ptr, self.n_state, self._ws_ptr,
                               self.ws.numel(), self.chunk, dt, self._P_ptr,
                               self.P.shape[0], 1, self.max_steps, self._model_ptr,
                               self.device.stream_ptr(sm))
            else:
                flags = abi.PSB_TAB_SHARED_V if (self.h_tables["flags"][ti] & abi.PSB_TAB_SHARED_V) else 0
                self._lib.call("psb_rk4_f64", *common, ptr, n_launch, self._y_ptr,
                               self.n_state, nk, flags, self.chunk, dt, self._P_ptr,
                               self.P.shape[0], 1, self.max_steps, self._model_ptr,
                               self.device.stream_ptr(sm))
            self.steps_done[slots] += self.chunk
            if fin.size:
                self._retire(lane, fin, st.view(r_fin, torch.int64), st.view(r_foff, torch.int64))
            ev = torch.cuda.Event()
            ev.record(sm)
        lane.inflight.append(ev)
        lane.tick += 1
        self.tick += 1
        return True

    def _retire(self, lane, fin, fin_t, foff_t):
        """Gather the finished solves' records, state and descriptors on the
        lane's stream (the current stream), then copy them to pinned host
        memory on the copy stream."""
        torch = self.torch
        # (slot, request, steps done, admission time, bytes)
        entries = []
        for g in fin:
            req, _, admitted, nbytes = self.active.pop(int(g))
            entries.append((int(g), req, int(self.steps_done[int(g)]), admitted, nbytes))
        lane.mask[fin - lane.base] = False
        lane.nactive -= len(fin)
        rows = self._rows(foff_t, lane.nk)
        # P(t) records up to the longest of these solves, not max_steps
        smax = max(e[1].nsteps for e in entries)
        Pg = self.P.view(self.nslots, self.max_steps, 2)[:, :smax].index_select(0, fin_t)
        yg = self.y.index_select(0, rows)
        wgr = self._wires_rows.index_select(0, fin_t)
        ev0 = torch.cuda.Event()
        ev0.record(torch.cuda.current_stream())
        cs = self.copy_stream
        cs.wait_event(ev0)
        # one pinned buffer from the pool for the three copies
        nP, ny = Pg.numel() * 8, yg.numel() * 8
        nbuf = nP + ny + wgr.numel()
        hbuf = self._pinned(nbuf)
        hP = hbuf[:nP].view(torch.float64).view(Pg.shape)
        hy = hbuf[nP:nP + ny].view(torch.float64).view(yg.shape)
        hw = hbuf[nP + ny:nbuf].view(wgr.shape)
        with torch.cuda.stream(cs):
            hP.copy_(Pg, non_blocking=True)
            hy.copy_(yg, non_blocking=True)
            hw.copy_(wgr, non_blocking=True)
            Pg.record_stream(cs)
            yg.record_stream(cs)
            wgr.record_stream(cs)
            ev = torch.cuda.Event()
            ev.record(cs)
        self.d2h_bytes += (hP.numel() + hy.numel()) * 8 + hw.numel()
        self.pending.append((ev, entries, (hP, hy, hw), hbuf))

    def _pinned(self, nbytes):
        """A pinned host byte buffer of at least nbytes: a collected one from
        the pool when one fits (at most 4x larger), else a new one of the
        next power of two (>= 1 MiB).  Sizes are multiples of 8, so float64
        views at 8-byte offsets stay aligned."""
        for i, buf in enumerate(self._pin_free):
            if nbytes <= buf.numel() <= 4 * max(nbytes, 1 << 20):
                return self._pin_free.pop(i)
        size = 1 << max(20, (int(nbytes) - 1).bit_length())
        return self.torch.empty(size, dtype=self.torch.uint8, pin_memory=True)

    def _collect(self, block=False):
        keep = []
        for item in self.pending:
            ev, entries, (hP, hy, hw), hbuf = item
            if block:
                ev.synchronize()
            elif not ev.query():
                keep.append(item)
                continue
            now = time.perf_counter() - self.t_start
            # one copy of each block out of the pinned buffer, which goes
            # back to the pool; every result is a view into these copies
            P, Y = hP.numpy().copy(), hy.numpy().copy()
            W = hw.numpy().reshape(-1).view(abi.WIRE_DTYPE).copy()
            self._pin_free.append(hbuf)
            st_all = W["status"].astype(np.int64)
            o = 0
            for i, (g, req, done, admitted, nbytes) in enumerate(entries):
                status, nsteps = int(st_all[i]), req.nsteps
                if req.rid in self._cancelled:
                    self._cancelled.discard(req.rid)
                    status, nsteps = STATUS_CANCELLED, min(req.nsteps, int(done))
                # P(t) rows (re, im) viewed as complex128
                p = P[i, :nsteps].view(np.complex128).reshape(-1)
                self.results.append(Result(req.rid, req.nk, nsteps, req.arrival, admitted, now,
                                           status, p, Y[o:o + req.nk]))
                o += req.nk
                self.pool.give_back(req.nk, g - self.cls_base[req.nk], nbytes)
        self.pending = keep

    def cancel(self, rid):
        """Cancel request ``rid``: a waiting request leaves its queue at once,
        a running one retires at its next tick boundary (its P(t) records and
        state up to there are returned); either way its Result has status
        STATUS_CANCELLED."""
        self._cancel.add(int(rid))

    def _apply_cancels(self, now):
        if not self._cancel:
            return
        for lane in self.lanes:
            keep = collections.deque()
            for req in lane.waiting:
                if req.rid in self._cancel:
                    self._cancel.discard(req.rid)
                    self.results.append(Result(req.rid, req.nk, 0, req.arrival, now, now,
                                               STATUS_CANCELLED, np.zeros(0, complex),
                                               np.zeros((0, 4))))
                else:
                    keep.append(req)
            lane.waiting = keep
        for g, entry in self.active.items():
            req = entry[0]
            if req.rid in self._cancel:
                self._cancel.discard(req.rid)
                self._cancelled.add(req.rid)
                # finish with the next tick: its end is the tick boundary
                self.steps_req[g] = min(self.steps_req[g], self.steps_done[g] + self.chunk)

    def run(self, requests, realtime=True, max_inflight_ticks=None, cancels=(),
            longest_first=None):
        """Serve ``requests``.  realtime: arrivals are honoured on the wall
        clock (the Poisson stream), else every request is available from the
        start (throughput / capacity runs).

        longest_first (default: not realtime): each size class admits its
        waiting solves longest first instead of in arrival order -- for a
        backlog this shortens the tail in which the last long solves run
        with few slots busy (longest-processing-time-first scheduling).  A
        solve's result does not depend on when it is admitted.

        Each size class ticks on its own stream as soon as its previous
        ticks allow (at most ``max_inflight_ticks`` queued), so a small
        solve advances at its own kernel's pace instead of waiting each tick
        for the largest grid; the classes' launches run concurrently on the
        GPU.  Largest grids are served first in each round.

        cancels: (time, rid) pairs; at that time (stream clock) ``cancel(rid)``
        is applied, as a client withdrawing a request would."""
        if max_inflight_ticks is None:
            max_inflight_ticks = self.max_inflight
        if longest_first is None:
            longest_first = not realtime
        assert max_inflight_ticks < self.ring
        queue = sorted(requests, key=lambda r: r.arrival)
        for req in queue:
            if req.nsteps > self.max_steps:
                raise ValueError(f"request {req.rid}: {req.nsteps} steps > max_steps")
            if req.nk not in self.cls_base:
                raise ValueError(f"request {req.rid}: Nk {req.nk} is not served")
        by_nk = {lane.nk: lane for lane in self.lanes}
        order = sorted(self.lanes, key=lambda ln: -ln.nk)
        qi, n = 0, len(queue)
        cq = sorted(cancels)
        ci = 0
        self.results = []
        self.t_start = time.perf_counter()
        while len(self.results) < n:
            now = time.perf_counter() - self.t_start
            arrived = qi
            while qi < n and (not realtime or queue[qi].arrival <= now):
                by_nk[queue[qi].nk].waiting.append(queue[qi])
                qi += 1
            if longest_first and qi > arrived:
                for lane in self.lanes:
                    if len(lane.waiting) > 1:
                        lane.waiting = collections.deque(
                            sorted(lane.waiting, key=lambda r: -r.nsteps))
            while ci < len(cq) and cq[ci][0] <= now:
                self.cancel(cq[ci][1])
                ci += 1
            self._apply_cancels(now)
            self._collect()
            issued = False
            for lane in order:
                while lane.inflight and lane.inflight[0].query():
                    lane.inflight.pop(0)
                if len(lane.inflight) < max_inflight_ticks and (lane.slots or lane.waiting):
                    issued |= self._tick(lane, now)
            if issued:
                continue
            busy = [ln.inflight[0] for ln in order if ln.inflight]
            if self.pending and not busy:
                self._collect(block=True)
            elif busy:
                time.sleep(5e-5)
            elif qi < n and realtime:
                time.sleep(max(0.0, min(1e-3, queue[qi].arrival - now)))
        self.torch.cuda.synchronize()
        self._collect(block=True)
        self._cancel.clear()
        self.elapsed = time.perf_counter() - self.t_start
        return sorted(self.results, key=lambda r: r.rid)

    def latency_percentiles(self, qs=(50, 99)):
        lat = np.array([r.latency for r in self.results])
        return {q: float(np.percentile(lat, q)) for q in qs} if lat.size else {}

    def throughput(self):
        """Completed wire*k*steps per second of the run."""
        work = sum(r.nk * r.nsteps for r in self.results)
        return work / self.elapsed if self.elapsed > 0 else 0.0


def wire_records(reqs, grid, table=0, offs=0, p_offs=0):
    """wire_record of many requests at once (elementwise the same arithmetic,
    so each record has the bits wire_record gives it)."""
    n = len(reqs)
    rec = np.zeros(n, dtype=abi.WIRE_DTYPE)
    det = np.array([r.det_eV for r in reqs], dtype=np.float64)
    T2 = np.array([r.T2 for r in reqs], dtype=np.float64)
    theta = np.array([r.theta for r in reqs], dtype=np.float64)
    fwhm = np.array([r.fwhm for r in reqs], dtype=np.float64)
    mscale = grid.ehint * grid.dcv / 2.0
    rec["table"] = table
    rec["npulse"] = 1
    rec["off"] = offs
    rec["gap"] = -det * EV
    rec["gamma"] = 1.0 / T2
    rec["mscale"] = mscale
    rec["pscale"] = grid.pscale
    from .grid import gaussian_amplitude

    rec["amp"][:, 0] = gaussian_amplitude(theta, fwhm, mscale)
    rec["t0"][:, 0] = 3.0 * fwhm
    rec["fwhm"][:, :] = fwhm[:, None]
    rec["p_off"] = p_offs
    return rec


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
