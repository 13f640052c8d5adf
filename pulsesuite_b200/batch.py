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
    def __init__(self, grids, wires, screened=False, excitons=True, p_cap=0, tables=None,
                 tabdata=None):
        device.require_cuda()
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
        # Largest grids first: balances uneven batches on the CTA scheduler.
        order = np.argsort(-nks, kind="stable").astype(np.int32)
        self.d_order = torch.as_tensor(order, device="cuda")
        self.model = abi.model_array(hbar)

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
    def rhs(self, stream=None):
        dy = torch.empty_like(self.y)
        _lib.call("psb_rhs_f64", *self._common(), device.ptr(self.y), device.ptr(dy),
                  self.n_state, self.nkmax, int(self.screened), abi.as_ptr(self.model),
                  device.stream_ptr(stream))
        return dy

    def rk4(self, nsteps, dt, p_stride=1, stream=None):
        _lib.call("psb_rk4_f64", *self._common(), device.ptr(self.d_order), device.ptr(self.y),
                  self.n_state, self.nkmax, int(self.screened), int(nsteps), float(dt),
                  device.ptr(self.P), self.P.shape[0], int(p_stride), self.p_cap,
                  abi.as_ptr(self.model), device.stream_ptr(stream))

    def leapfrog(self, field, nsteps, dt, p_stride=1, stream=None):
        """field: device float64 tensor (nw, 2*n_samples) of sampled E(t_n)."""
        if self.y1 is None:
            self.y1 = self.y.clone()
        assert field.is_cuda and field.dtype == torch.float64 and field.dim() == 2
        _lib.call("psb_leapfrog_f64", *self._common(), device.ptr(self.d_order),
                  device.ptr(self.y1), device.ptr(self.y), self.n_state, self.nkmax,
                  int(self.screened), device.ptr(field), field.shape[1], field.numel(),
                  int(nsteps), float(dt), device.ptr(self.P), self.P.shape[0], int(p_stride),
                  self.p_cap, abi.as_ptr(self.model), device.stream_ptr(stream))
