"""Batched quantum-wire SBE engine: many wires of uneven k grids resident on
one GPU, advanced by the fused sm_100a step kernels.

    b = WireBatch(grids, wires, screened=False)
    P = b.rk4(nsteps, dt, p_stride=1)      # P(t) records, device tensor
    y = b.state()                           # (n_state, 4) float64 on the host

``wires`` is a numpy array of ``abi.WIRE_DTYPE``; ``table`` indexes
``grids``.  The batch assigns the state (``off``) and P(t) (``p_off``)
ranges.  Buffers are torch tensors on the current device; the step entry
points allocate nothing.
"""

import numpy as np
import torch
from scipy.constants import hbar

from . import _lib, abi, coulomb, device


class WireBatch:
    """``form`` selects the step kernel: "plain" (FP64 throughout,
    psb_rk4_f64) or "split" (exchange sums on the int8 tensor cores as exact
    products of base-254 digits, FP64 right-hand side and state:
    psb_rk4_split for unscreened grids with one shared Coulomb matrix,
    psb_rk4_split_wire for screened grids or distinct Veh, Vee, Vhh)."""

    def __init__(self, grids, wires, screened=False, excitons=True, p_cap=0, tables=None,
                 tabdata=None, form="plain", split_w=None, tune=True):
        device.require_cuda()
        if form not in ("plain", "split"):
            raise ValueError("form must be 'plain' or 'split'")
        self.form = form
        # split form: wires per CTA group by grid size, {nk: 4, 8 or 16}; grids
        # not listed use the built-in rule (see _setup_split)
        self.split_w = dict(split_w or {})
        self.tune = bool(tune)
        self.grids = list(grids)
        self.screened = bool(screened)
        if tables is None:
            tables, tabdata = coulomb.grid_tables(self.grids, screened=screened,
                                                  excitons=excitons)
        self.h_tables = np.ascontiguousarray(tables)
        self.tabdata = tabdata
        self.nkmax = int(self.h_tables["nk"].max())
        w = np.array(wires, dtype=abi.WIRE_DTYPE, copy=True)
        nks = self.h_tables["nk"][w["table"]].astype(np.int64)
        offs = np.zeros(len(w), dtype=np.int64)
        if len(w):
            offs[1:] = np.cumsum(nks)[:-1]
        w["off"] = offs
        self.p_cap = int(p_cap)
        w["p_off"] = np.arange(len(w), dtype=np.int64) * self.p_cap
        self.nks = nks
        self.n_state = int(nks.sum())
        self.nw = len(w)
        self.h_wires = w
        self.d_tables = device.to_device(self.h_tables)
        self.d_wires = device.to_device(w)
        self.y = torch.zeros((self.n_state, 4), dtype=torch.float64, device="cuda")
        self.y1 = None
        self.P = torch.zeros((max(1, self.nw * self.p_cap), 2), dtype=torch.float64,
                             device="cuda")
        # Launch classes by grid size (registers and shared memory are sized
        # for a class's largest grid); largest grids first inside a class
        # balances uneven batches on the CTA scheduler.
        self.classes = []
        order = np.argsort(-nks, kind="stable").astype(np.int32)
        for lo, hi in ((0, 256), (256, 512), (512, abi.PSB_MAX_NK)):
            sel = order[(nks[order] > lo) & (nks[order] <= hi)]
            if sel.size == 0:
                continue
            tabs = np.unique(w["table"][sel])
            tf = self.h_tables["flags"][tabs]
            flags = 0
            if (tf & abi.PSB_TAB_SCREENED).any():
                flags |= abi.PSB_TAB_SCREENED
            if (tf & abi.PSB_TAB_SHARED_V).all():
                flags |= abi.PSB_TAB_SHARED_V
            self.classes.append((torch.as_tensor(sel, device="cuda"), int(nks[sel].max()), flags))
        if form == "split":
            self._setup_split()
        self.tab_flags = 0
        if (self.h_tables["flags"] & abi.PSB_TAB_SCREENED).any():
            self.tab_flags |= abi.PSB_TAB_SCREENED
        if (self.h_tables["flags"] & abi.PSB_TAB_SHARED_V).all():
            self.tab_flags |= abi.PSB_TAB_SHARED_V
        self.model = abi.model_array(hbar)

    def _setup_split(self):
        """Wire groups (one CTA each) and the workspace of the split form.

        Unscreened grids with Veh == Vee == Vhh use psb_rk4_split: a group
        holds up to W in {4, 8, 16} wires of one grid sharing one Coulomb
        matrix.  W is chosen per grid by the autotuner (tune.SplitTuner:
        measured per-CTA cost of each W on this device, times the waves of
        CTAs the grid's wire count needs); with ``tune=False`` by a rule
        (W = 8 once a grid has enough wires for roughly two waves of CTAs,
        else 4); ``split_w`` overrides both per grid.  Groups are launched in
        classes of (W, state resident in shared memory or not) so that a
        large grid does not push the small ones out of the resident layout.

        Screened grids and grids with distinct Veh, Vee, Vhh use
        psb_rk4_split_wire (one matrix per wire, the wires of a group
        contracted one after another): W is the largest group that fits, but
        no more wires per CTA than a full wave of CTAs leaves
        (``split_w`` overrides it, 1 .. psb_split_wire_max_group).

        All classes run concurrently on side streams, the one with the
        largest grid first."""
        f = self.h_tables["flags"]
        if ((f & abi.PSB_TAB_EXCITONS) == 0).any():
            raise _lib.PsbError("split form needs tables with excitons (the exchange sums)")
        lib = _lib.load()
        maxnk = {wg: int(lib.psb_split_max_nk(wg)) for wg in (4, 8, 16)}
        resnk = {wg: int(lib.psb_split_max_nk_resident(wg)) for wg in (4, 8, 16)}
        nks = self.h_tables["nk"].astype(np.int64)
        counts = np.bincount(self.h_wires["table"], minlength=len(nks))
        sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        target = float(np.sum(counts * nks.astype(np.float64) ** 2)) / (2.0 * sms)
        classes = {}
        wclasses = {}
        for t in np.argsort(-nks, kind="stable"):
            nk = int(nks[t])
            if counts[t] == 0:
                continue
            ws = np.nonzero(self.h_wires["table"] == t)[0]
            tflags = int(f[t]) & (abi.PSB_TAB_EXCITONS | abi.PSB_TAB_SCREENED |
                                  abi.PSB_TAB_SHARED_V)
            per_wire = (tflags & abi.PSB_TAB_SCREENED) or not (tflags & abi.PSB_TAB_SHARED_V)
            if per_wire:
                wmax = int(lib.psb_split_wire_max_group(nk, tflags))
                if wmax < 1:
                    raise _lib.PsbError(f"split form: nk {nk} exceeds the supported maximum "
                                        "for screened or distinct Coulomb matrices")
                wg = max(1, min(wmax, -(-len(ws) // sms)))
                if nk in self.split_w:
                    wg = int(self.split_w[nk])
                    if not 1 <= wg <= wmax:
                        raise ValueError(f"split_w[{nk}] must be 1..{wmax} for these tables")
                key = (wg, tflags)
                target_classes = wclasses
            else:
                wg = 4
                if self.tune:
                    from .tune import shared_tuner

                    wg = shared_tuner().best_width(nk, int(counts[t]))
                elif nk <= maxnk[8] and 8 * nk * nk <= max(target, 4 * nk * nk):
                    wg = 8
                if nk in self.split_w:
                    wg = int(self.split_w[nk])
                    if wg not in (4, 8, 16):
                        raise ValueError("split_w values must be 4, 8 or 16")
                if nk > maxnk[wg]:
                    raise _lib.PsbError(f"split form: nk {nk} exceeds the supported maximum")
                key = (wg, nk <= resnk[wg])
                target_classes = classes
            for i in range(0, len(ws), wg):
                g = np.zeros(1, dtype=abi.SPLIT_GROUP_DTYPE)
                g["table"] = t
                g["nw"] = len(ws[i:i + wg])
                g["wire"][0, :] = -1
                g["wire"][0, :g["nw"][0]] = ws[i:i + wg]
                target_classes.setdefault(key, []).append(g)
        self.split_launches = []
        for key in classes:
            ga = np.concatenate(classes[key])
            nkmax = int(nks[ga["table"]].max())
            self.split_launches.append((key[0], device.to_device(ga), len(ga), nkmax))
        # the class with the largest grid first: its CTAs run longest
        self.split_launches.sort(key=lambda l: -l[3])
        # per-wire classes: (W, groups, count, nkmax, table flags)
        self.wire_launches = []
        for key in wclasses:
            ga = np.concatenate(wclasses[key])
            nkmax = int(nks[ga["table"]].max())
            self.wire_launches.append((key[0], device.to_device(ga), len(ga), nkmax, key[1]))
        self.wire_launches.sort(key=lambda l: -l[3])
        # one stream per class, priorities by grid size (the largest grid's
        # CTAs run longest, so the CTA scheduler serves them first)
        least, greatest = torch.cuda.Stream.priority_range()
        nl = len(self.split_launches) + len(self.wire_launches)
        self.side_streams = [torch.cuda.Stream(priority=min(least, greatest + r))
                             for r in range(nl)]
        self.ws = torch.zeros(int(lib.psb_split_ws_bytes(self.n_state)), dtype=torch.uint8,
                              device="cuda")

    # -- state --------------------------------------------------------------
    def set_state(self, y, y1=None):
        self.y.copy_(torch.as_tensor(np.asarray(y, dtype=np.float64).reshape(self.n_state, 4)))
        if y1 is not None:
            if self.y1 is None:
                self.y1 = torch.zeros_like(self.y)
            self.y1.copy_(torch.as_tensor(np.asarray(y1, dtype=np.float64).reshape(-1, 4)))

    def state(self):
        return self.y.cpu().numpy()

    def wires(self):
        """Current wire descriptors (t, steps, status) from the device."""
        return device.to_host_struct(self.d_wires, abi.WIRE_DTYPE)

    def wire_slice(self, i):
        o = int(self.h_wires["off"][i])
        return slice(o, o + int(self.nks[i]))

    def records(self, i):
        """P(t) records of wire i as complex numpy."""
        P = self.P[i * self.p_cap:(i + 1) * self.p_cap].cpu().numpy()
        return P[:, 0] + 1j * P[:, 1]

    def _common(self):
        return (device.ptr(self.d_tables), len(self.h_tables), device.ptr(self.tabdata),
                self.tabdata.numel(), device.ptr(self.d_wires), self.nw)

    # -- entry points -----------------------------------------------------------
    @property
    def launches_per_call(self):
        """Kernel launches one rk4/leapfrog call issues (one per size class)."""
        if self.form == "split":
            return len(self.split_launches) + len(self.wire_launches)
        return len(self.classes)

    def rhs(self, stream=None):
        dy = torch.empty_like(self.y)
        _lib.call("psb_rhs_f64", *self._common(), device.ptr(self.y), device.ptr(dy),
                  self.n_state, self.nkmax, self.tab_flags, abi.as_ptr(self.model),
                  device.stream_ptr(stream))
        return dy

    def rk4(self, nsteps, dt, p_stride=1, stream=None):
        if self.form == "split":
            main = stream if stream is not None else torch.cuda.current_stream()
            streams = self.side_streams
            fork = torch.cuda.Event()
            fork.record(main)
            for s in streams:
                s.wait_event(fork)
            for (wg, groups, ng, nkmax), s in zip(self.split_launches, streams):
                _lib.call("psb_rk4_split", *self._common(), device.ptr(groups), ng, wg, nkmax,
                          device.ptr(self.y), self.n_state, device.ptr(self.ws), self.ws.numel(),
                          int(nsteps), float(dt), device.ptr(self.P), self.P.shape[0],
                          int(p_stride), self.p_cap, abi.as_ptr(self.model),
                          device.stream_ptr(s))
            for (wg, groups, ng, nkmax, tflags), s in zip(self.wire_launches,
                                                         streams[len(self.split_launches):]):
                _lib.call("psb_rk4_split_wire", *self._common(), device.ptr(groups), ng, wg,
                          nkmax, tflags, device.ptr(self.y), self.n_state, device.ptr(self.ws),
                          self.ws.numel(), int(nsteps), float(dt), device.ptr(self.P),
                          self.P.shape[0], int(p_stride), self.p_cap, abi.as_ptr(self.model),
                          device.stream_ptr(s))
            for s in streams:
                join = torch.cuda.Event()
                join.record(s)
                main.wait_event(join)
            return
        for order, nkmax, flags in self.classes:
            _lib.call("psb_rk4_f64", *self._common(), device.ptr(order), order.numel(),
                      device.ptr(self.y), self.n_state, nkmax, flags, int(nsteps), float(dt),
                      device.ptr(self.P), self.P.shape[0], int(p_stride), self.p_cap,
                      abi.as_ptr(self.model), device.stream_ptr(stream))

    def capture(self, nsteps, dt, p_stride=1):
        """A CUDA graph of one ``rk4(nsteps, dt, p_stride)`` call (every size
        class's launch, the split form's side streams and their joins), to
        replay with ``graph.replay()`` on the current stream: one host call
        per step instead of one launch per class plus the stream
        synchronisation.  The graph reads and writes this batch's own state,
        wire descriptors and P(t) buffers, so a caller changes the data
        between replays (``set_state``, the wire descriptors), not the
        shapes.  One eager call first sets the kernels' attributes outside
        the capture (it advances the batch like any rk4 call)."""
        import torch

        self.rk4(nsteps, dt, p_stride=p_stride)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.rk4(nsteps, dt, p_stride=p_stride)
        torch.cuda.synchronize()
        return g

    def leapfrog(self, field, nsteps, dt, p_stride=1, stream=None):
        """field: device float64 tensor (nw, 2*n_samples) of sampled E(t_n)."""
        if self.y1 is None:
            self.y1 = self.y.clone()
        assert field.is_cuda and field.dtype == torch.float64 and field.dim() == 2
        for order, nkmax, flags in self.classes:
            _lib.call("psb_leapfrog_f64", *self._common(), device.ptr(order), order.numel(),
                      device.ptr(self.y1), device.ptr(self.y), self.n_state, nkmax, flags,
                      device.ptr(field), field.shape[1], field.numel(), int(nsteps), float(dt),
                      device.ptr(self.P), self.P.shape[0], int(p_stride), self.p_cap,
                      abi.as_ptr(self.model), device.stream_ptr(stream))
