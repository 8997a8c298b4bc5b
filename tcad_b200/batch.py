"""Many devices of one dimension solved together on one GPU.

The devices' arrays are packed back to back into one HBM pack
(include/tcad_b200.h); every kernel launch covers every instance, and the
Newton and Krylov drivers keep per-instance scalars and convergence masks, so
finished instances drop out of the launched work while the others continue.
Each instance's result is the one it gets when solved alone (the
per-instance reductions never mix instances).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .options import NewtonOptions
from .pack import Pack, bias_vector, secant_ratio


class DeviceBatch:
    """A packed batch of Device2D (or Device3D) instances.

    The member devices keep their own contacts and gates; their numpy state
    attributes are not used while they are batched (read results through
    ``state(i)`` and ``terminal_currents``)."""

    def __init__(self, devices):
        self.devices = list(devices)
        dims = {d.dim for d in self.devices}
        if len(dims) != 1:
            raise ValueError("a batch holds devices of one dimension")
        self.pack = Pack([d.setup for d in self.devices])
        self.n = len(self.devices)
        self.have_state = np.zeros(self.n, dtype=bool)
        self.bias_prev = [None] * self.n     # per instance: bias of the prev / current state
        self.bias_cur = [None] * self.n
        self.last = None
        self._guess = None   # bulk-guess potential, resident after first use

    def _ctypes_voltages(self, voltages):
        if voltages is None:
            return
        if len(voltages) != self.n:
            raise ValueError("one voltage dict per instance")
        for dev, volts in zip(self.devices, voltages):
            dev._apply_voltages(volts)

    def solve_equilibrium(self, opts: NewtonOptions = None):
        """Equilibrium Poisson for every instance (one packed solve)."""
        opts = opts or NewtonOptions()
        pk = self.pack
        if self._guess is None:
            guess = np.concatenate([d.setup.bulk_guess().ravel() for d in self.devices])
            self._guess = pk.torch.from_numpy(guess).to(pk.device)
        pk.psi.copy_(self._guess)
        res = pk.equilibrium(opts)
        self.have_state[:] = True
        self.bias_prev = [None] * self.n
        self.bias_cur = [np.zeros(len(d.bcs)) for d in self.devices]
        self.last = res
        return res

    def solve_bias(self, voltages=None, opts: NewtonOptions = None, active=None):
        """Coupled Newton at each instance's own bias (voltages: list of
        per-instance {name: V} dicts); instances with active[i] False keep
        their state.  Returns the per-instance Newton results."""
        opts = opts or NewtonOptions()
        if not self.have_state.all():
            self.solve_equilibrium(opts)
        self._ctypes_voltages(voltages)
        pk = self.pack
        pk.set_bias()
        act = np.ones(self.n, dtype=bool) if active is None else np.asarray(active, bool)
        new = [bias_vector(d.setup) for d in self.devices]
        use_pred = getattr(opts, "predictor", "none") == "secant"
        ratios = [secant_ratio(self.bias_prev[i], self.bias_cur[i], new[i])
                  if (use_pred and act[i]) else 0.0 for i in range(self.n)]
        if use_pred:
            # inactive instances: ratio 0 (their state is saved, not moved)
            pk.predict(ratios)
        pk.stamp_contacts(active)
        res = pk.newton(opts, active=active)
        retry = [i for i in range(self.n) if act[i] and ratios[i] != 0.0
                 and not res[i]["converged"]]
        if retry:
            pk.restore_prev(retry)
            mask = np.zeros(self.n, dtype=bool)
            mask[retry] = True
            pk.stamp_contacts(mask)
            res2 = pk.newton(opts, active=mask)
            for i in retry:
                r = res2[i]
                r["iters"] += res[i]["iters"]
                r["krylov_iters"] += res[i]["krylov_iters"]
                r["predictor_retry"] = True
                res[i] = r
        for i in range(self.n):
            if not act[i]:
                if use_pred:       # its prev buffer now holds its current state
                    self.bias_prev[i] = None
                continue
            self.bias_prev[i] = self.bias_cur[i] if use_pred else None
            self.bias_cur[i] = new[i] if res[i]["converged"] else None
        self.last = res
        return res

    def terminal_currents(self, name):
        """Contact current of every instance: A/cm (2D) or A (3D)."""
        out = np.zeros(self.n)
        exp = 1 if self.devices[0].dim == 2 else 2
        for i, d in enumerate(self.devices):
            I = float(self.pack.contact_current(i, name).item())
            out[i] = I * d.J0 * d.LD ** exp
        return out

    def state(self, i):
        """(psi, n, p) of instance i, shaped like the device's node grid."""
        pk = self.pack
        a, b = int(pk.node_off[i]), int(pk.node_off[i + 1])
        shp = self.devices[i].setup.shape
        return tuple(t[a:b].cpu().numpy().reshape(shp) for t in (pk.psi, pk.n, pk.p))
