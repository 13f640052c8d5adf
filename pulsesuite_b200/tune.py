"""Autotuner of the split-form launch shape, keyed on (Nk, B).

The split kernel (``psb_rk4_split``) runs one CTA per group of W wires of
one k grid, W in {4, 8, 16}.  A wider group makes every tensor-core MMA
wider at the same issue cost, but also gives its CTA W times the
drain/epilogue work and fewer CTAs to fill the SMs; which W is fastest
depends on the grid size Nk (shared-memory residency, MMA vs epilogue
balance) and on how many wires B share the grid (waves of CTAs).

``SplitTuner`` measures, on the current device, the time of one CTA per
time step for each (Nk, W) on a full wave of CTAs (one CTA per SM), caches
it (in memory and in a JSON file keyed by device and library build), and
chooses:

  * ``best_width(nk, count)``: the W that advances ``count`` wires of one
    grid fastest, from the measured per-CTA cost and the number of waves
    ceil(ceil(count / W) / SMs) (the batch engine's choice per grid);
  * ``choose(counts)``: W per grid for one serving tick in which several
    grids share the SMs, minimising the estimated tick time
    max(longest CTA, total CTA time / SMs) (the server's choice).

Results of the kernel do not depend on W (each wire's arithmetic is the same
in any group), so the choice only moves time.
"""

import json
import math
import os

import numpy as np

WIDTHS = (4, 8, 16)


def _cache_file():
    return os.environ.get("PSB_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "pulsesuite_b200",
                                       "split_tune.json"))


def choose_widths(counts, sms, cost, allowed):
    """Greedy joint choice of W per grid for one tick (largest grids first):
    start from the narrowest allowed width and widen a grid while that
    shortens the estimated tick max(longest CTA, total / sms) (ties broken
    by less total CTA time, i.e. more SM time for the others)."""
    ws = {nk: min(allowed(nk)) for nk, c in counts.items() if c}
    if not ws:
        return ws

    def tick(wm):
        total = sum(-(-counts[nk] // wm[nk]) * cost(nk, wm[nk]) for nk in wm)
        return (max(max(cost(nk, wm[nk]) for nk in wm), total / sms), total)

    best = tick(ws)
    for nk in sorted(ws, reverse=True):
        for w in sorted(allowed(nk)):
            if w <= ws[nk]:
                continue
            trial = dict(ws)
            trial[nk] = w
            t = tick(trial)
            if t < best:
                ws, best = trial, t
    return ws


class SplitTuner:
    """Measured per-CTA cost of the split kernel by (Nk, W) on this device."""

    def __init__(self, steps=20, use_file=True):
        from . import _lib, device

        device.require_cuda()
        import torch

        self.torch = torch
        self.lib = _lib.load()
        self.steps = int(steps)
        props = torch.cuda.get_device_properties(torch.cuda.current_device())
        self.sms = props.multi_processor_count
        st = os.stat(_lib.LIB_PATH)
        self.key = f"{props.name}|sm{props.major}{props.minor}|{self.sms}|{st.st_size}|" \
                   f"{int(st.st_mtime)}|steps{self.steps}"
        self.maxnk = {w: int(self.lib.psb_split_max_nk(w)) for w in WIDTHS}
        self.cta_ms = {}
        self.use_file = use_file
        self.measured = 0
        if use_file:
            self._load()

    # -- cache ---------------------------------------------------------------
    def _load(self):
        try:
            with open(_cache_file()) as f:
                data = json.load(f).get(self.key, {})
            self.cta_ms = {tuple(int(x) for x in k.split(",")): float(v) for k, v in data.items()}
        except (OSError, ValueError):
            self.cta_ms = {}

    def _save(self):
        if not self.use_file:
            return
        path = _cache_file()
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            try:
                with open(path) as f:
                    data = json.load(f)
            except (OSError, ValueError):
                data = {}
            data[self.key] = {f"{nk},{w}": v for (nk, w), v in self.cta_ms.items()}
            tmp = path + f".{os.getpid()}"
            with open(tmp, "w") as f:
                json.dump(data, f)
            os.replace(tmp, path)
        except OSError:
            pass

    # -- measurement ---------------------------------------------------------------
    def allowed(self, nk):
        return tuple(w for w in WIDTHS if nk <= self.maxnk[w])

    def _measure(self, nk, w):
        """ms of one CTA per time step: a full wave (one CTA per SM) of
        groups of w wires of grid nk, timed with CUDA events on a launch of
        `steps` steps after one warm-up launch."""
        torch = self.torch
        from scipy.constants import hbar

        from . import abi, coulomb, device
        from . import grid as pgrid

        g = pgrid.wire_grid(nk)
        tables, tabdata = coulomb.grid_tables([g])
        nw = self.sms * w
        wires = np.zeros(nw, dtype=abi.WIRE_DTYPE)
        mscale = g.ehint * g.dcv / 2.0
        wires["npulse"] = 1
        wires["gamma"] = 1.0 / 150e-15
        wires["mscale"] = mscale
        wires["pscale"] = g.pscale
        wires["amp"][:, 0] = pgrid.gaussian_amplitude(np.pi, 60e-15, mscale)
        wires["t0"][:, 0] = 180e-15
        wires["fwhm"][:, :] = 60e-15
        wires["off"] = np.arange(nw, dtype=np.int64) * nk
        groups = np.zeros(self.sms, dtype=abi.SPLIT_GROUP_DTYPE)
        groups["table"] = 0
        groups["nw"] = w
        groups["wire"] = -1
        groups["wire"][:, :w] = np.arange(nw, dtype=np.int32).reshape(self.sms, w)
        d_tab, d_w, d_g = (device.to_device(a) for a in (tables, wires, groups))
        n_state = nw * nk
        y = torch.zeros((n_state, 4), dtype=torch.float64, device="cuda")
        ws = torch.empty(int(self.lib.psb_split_ws_bytes(n_state)), dtype=torch.uint8,
                         device="cuda")
        P = torch.zeros((1, 2), dtype=torch.float64, device="cuda")
        model = abi.model_array(hbar)
        stream = torch.cuda.current_stream()

        def launch():
            from . import _lib

            _lib.call("psb_rk4_split", device.ptr(d_tab), 1, device.ptr(tabdata), tabdata.numel(),
                      device.ptr(d_w), nw, device.ptr(d_g), self.sms, w, nk, device.ptr(y),
                      n_state, device.ptr(ws), ws.numel(), self.steps, 1e-15, device.ptr(P), 1,
                      1, 0, abi.as_ptr(model), device.stream_ptr(stream))

        launch()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        best = float("inf")
        for _ in range(2):
            e0.record(stream)
            launch()
            e1.record(stream)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        self.measured += 1
        return best / self.steps

    def cost(self, nk, w):
        """ms of one CTA of w wires of grid nk per time step (measured once,
        cached)."""
        key = (int(nk), int(w))
        if key not in self.cta_ms:
            self.cta_ms[key] = self._measure(*key)
            self._save()
        return self.cta_ms[key]

    def table(self, nks):
        """Measure every allowed (nk, W) of the given grids."""
        for nk in nks:
            for w in self.allowed(nk):
                self.cost(nk, w)
        return dict(self.cta_ms)

    # -- choices -----------------------------------------------------------------
    def best_width(self, nk, count):
        """W advancing `count` wires of grid nk in the least time: waves of
        CTAs times the per-CTA cost."""
        def t(w):
            ctas = -(-int(count) // w)
            return math.ceil(ctas / self.sms) * self.cost(nk, w)

        return min(self.allowed(nk), key=lambda w: (t(w), -w))

    def choose(self, counts):
        """W per grid for one serving tick (see module docstring)."""
        return choose_widths(counts, self.sms, self.cost, self.allowed)


_shared = None


def shared_tuner():
    """The process-wide tuner (its measurements are reused by every batch)."""
    global _shared
    if _shared is None:
        _shared = SplitTuner()
    return _shared
