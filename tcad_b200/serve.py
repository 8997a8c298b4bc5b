"""Continuous-batching solve service over an HBM-resident arena.

A request is a device (its host ``Setup`` with contacts and gates) plus a
list of bias points: one target reached by a short ramp, or an Id-V sweep.
The service keeps every admitted device resident on the GPU -- coefficients,
boundary-condition arrays, the Jacobian's fixed node-block pattern and the
last converged (psi, n, p) -- in one arena of node arrays per dimension, so
a sweep's next point warm-starts from its previous one and a repeated device
is not uploaded again.

Scheduling is continuous batching at bias-point granularity.  Each round
solves the next point of every in-flight request in ONE batched Newton solve
(``tcad_newton_solve`` over a pack whose tables list just those devices, at
their arena places: the kernels index node arrays by arena position, so
joining or leaving moves no device data).  Requests that arrive while a round
runs are admitted at the next round boundary if the arena has room (first
fit; idle resident devices are evicted least-recently-used first), so new
work joins work already on the GPU.  2D and 3D devices live in separate
arenas served by separate threads on separate CUDA streams, whose rounds run
concurrently on the device.

Per-instance reductions and convergence masks keep instances independent:
a request's result is the one it gets alone.
"""
from __future__ import annotations

import collections
import copy
import threading
import time

import numpy as np

from . import _lib
from .options import NewtonOptions
from .pack import (BC_ARRAYS, NODE_ARRAYS, Pack, axis_arrays, bc_node_arrays, bias_vector,
                   gate_map, instance_tables, instance_tiles, node_arrays, secant_ratio)

# 3D tile depth of resident devices: rounds mix device sizes, so one fixed
# depth; the measured optimum is 1-2 planes below ~1M nodes (4 only on 8M)
TILE_Z = 2

ALIGN = 32          # region starts on 32-node (256-byte) boundaries


def bytes_per_node(dim):
    """HBM bytes one resident node costs: coefficients, BC arrays, state, F,
    the node-block Jacobian, the Newton update and the Krylov workspace
    (FP64 BiCGStab vectors and the FP32 extension of the mixed-precision
    path), the ILU(0) preconditioner, the equilibrium PCG's red-black
    extension, and the previous state the sweep predictor extrapolates
    from."""
    ne = _lib.NE[dim]
    doubles = len(NODE_ARRAYS) + 3 * dim + len(BC_ARRAYS) + 3 + 3 + 3 + ne + 3
    work64 = 6 * 3 * 8 + 4 * 8 / 256
    work32 = 6 * 3 * 4 + ne * 4 + 2 * 3 * 4
    ilu = (9 + 6) * 8                        # ILU(0) factor and two vectors
    if dim == 2:                             # slot-order sweep data (FP32) and vectors
        ilu += 2 * (27 + 18) * 4 + 2 * 2 * 3 * 8
    eq = (2 * (1 + 2 * dim) + 5) * 8 + 2 * 4 / 256   # equilibrium red-black extension
    return int(np.ceil(doubles * 8 + 1 + work64 + work32 + ilu + eq))


class RangeAllocator:
    """First-fit allocator of ranges in [0, capacity), coalescing on release."""

    def __init__(self, capacity, align=1, start=0):
        self.capacity = int(capacity)
        self.align = int(align)
        self.free = [(int(start), self.capacity - int(start))] if capacity > start else []

    def _round(self, n):
        return -(-int(n) // self.align) * self.align

    def alloc(self, n):
        n = self._round(n)
        for i, (a, ln) in enumerate(self.free):
            if ln >= n:
                if ln == n:
                    del self.free[i]
                else:
                    self.free[i] = (a + n, ln - n)
                return a
        return None

    def release(self, a, n):
        n = self._round(n)
        free = self.free
        i = 0
        while i < len(free) and free[i][0] < a:
            i += 1
        free.insert(i, (a, n))
        # coalesce with the right, then the left neighbour
        if i + 1 < len(free) and free[i][0] + free[i][1] == free[i + 1][0]:
            free[i] = (free[i][0], free[i][1] + free[i + 1][1])
            del free[i + 1]
        if i > 0 and free[i - 1][0] + free[i - 1][1] == free[i][0]:
            free[i - 1] = (free[i - 1][0], free[i - 1][1] + free[i][1])
            del free[i]

    def free_total(self):
        return sum(ln for _, ln in self.free)

    def largest(self):
        return max((ln for _, ln in self.free), default=0)


class Placement:
    """Where a resident device lives in its arena, and its cached tables."""

    def __init__(self, off, n, axis_off, axis_len, tiles, ctab, gm, gnodes, h2d):
        self.off, self.n = off, n
        self.axis_off, self.axis_len = axis_off, axis_len
        self.tiles, self.ctab = tiles, ctab
        self.gm, self.gnodes = gm, gnodes
        self.h2d_bytes = h2d


class Arena:
    """Node arrays of one dimension sized for a byte budget; devices are
    placed in ranges of them (first fit) and stay until released."""

    def __init__(self, dim, budget_bytes, device="cuda", max_inst=4096):
        import torch
        self.torch = torch
        self.dim = dim
        self.device = torch.device(device)
        self.lib = _lib.load()
        cap = int(budget_bytes) // bytes_per_node(dim)
        self.cap = cap = max(ALIGN, cap // ALIGN * ALIGN)
        self.max_inst = int(max_inst)
        f64 = dict(dtype=torch.float64, device=self.device)
        t = {}
        for name in NODE_ARRAYS + BC_ARRAYS:
            t[name] = torch.zeros(cap, **f64)
        for a in range(dim):
            for name in ("an", "ap", "dl"):
                t[f"{name}{a}"] = torch.zeros(cap, **f64)
        t["bcflag"] = torch.zeros(cap, dtype=torch.uint8, device=self.device)
        # per-axis entries: index 0 holds the (h=0, dv=1) filler of unused axes
        self.axcap = max(1 << 16, cap // 8)
        for a in range(3):
            t[f"h{a}"] = torch.zeros(self.axcap, **f64)
            t[f"dv{a}"] = torch.ones(self.axcap, **f64)
        self.t = t
        self.psi, self.n, self.p = (torch.zeros(cap, **f64) for _ in range(3))
        self.prev = tuple(torch.zeros(cap, **f64) for _ in range(3))
        self.F = torch.zeros(3 * cap, **f64)
        self.J = torch.zeros(_lib.NE[dim] * cap, **f64)
        self.du = torch.zeros(3 * cap, **f64)
        P = _lib.TcadPack()
        P.dim = dim
        P.n_inst = self.max_inst
        P.n_nodes = cap
        P.n_flat = cap // 256 + self.max_inst    # any flat_nodes >= 256
        P.flat_nodes = _lib.FLAT_NODES
        P.tile_z = TILE_Z
        # sized without the red-black extension (method 0): served solves run
        # on the whole system -- the mixed-precision default does anyway --
        # and the arena keeps its nodes for devices
        wb = int(self.lib.tcad_block_workspace_bytes(ctypes_ref(P), 0, 0))
        self.work = torch.empty(wb, dtype=torch.uint8, device=self.device)
        self.nodes = RangeAllocator(cap, ALIGN)
        self.axes = [RangeAllocator(self.axcap, 1, start=1) for _ in range(3)]
        self.lock = threading.Lock()

    def hbm_bytes(self):
        tot = sum(v.numel() * v.element_size() for v in self.t.values())
        for v in (self.psi, self.n, self.p, self.F, self.J, self.du, self.work) + self.prev:
            tot += v.numel() * v.element_size()
        return tot

    def fits(self, setup):
        return setup.N <= self.nodes.largest()

    def place(self, setup):
        """Allocate a range for the device and upload its arrays (on the
        current stream).  Returns None when the arena has no room."""
        torch = self.torch
        dim = self.dim
        with self.lock:
            off = self.nodes.alloc(setup.N)
            if off is None:
                return None
            axes = axis_arrays(setup, dim)
            axis_off = np.zeros(3, dtype=np.int64)
            got = []
            for a in range(dim):
                o = self.axes[a].alloc(axes[a][1].size)
                if o is None:
                    for b, ob in got:
                        self.axes[b].release(ob, axes[b][1].size)
                    self.nodes.release(off, setup.N)
                    return None
                got.append((a, o))
                axis_off[a] = o
        h2d = 0

        def put(name, arr, lo, dtype=None):
            nonlocal h2d
            src = torch.from_numpy(np.ascontiguousarray(arr))
            if dtype is not None:
                src = src.to(dtype)
            self.t[name][lo:lo + src.numel()].copy_(src)
            h2d += src.numel() * src.element_size()

        for a in range(dim):
            put(f"h{a}", axes[a][0], int(axis_off[a]))
            put(f"dv{a}", axes[a][1], int(axis_off[a]))
        for name, arr in node_arrays(setup).items():
            put(name, arr, off)
        arrs, ctab = bc_node_arrays(setup)
        for name, arr in arrs.items():
            put(name, arr, off)
        for name in ("bc_psi0", "bc_n0", "bc_p0"):
            self.t[name][off:off + setup.N].zero_()
        guess = setup.bulk_guess().ravel()
        self.psi[off:off + setup.N].copy_(torch.from_numpy(guess))
        h2d += guess.nbytes
        gm, gnodes = gate_map(setup)
        return Placement(off, setup.N, axis_off, [axes[a][1].size for a in range(3)],
                         instance_tiles(setup, dim, TILE_Z), ctab, gm, gnodes, h2d)

    def release(self, pl):
        with self.lock:
            self.nodes.release(pl.off, pl.n)
            for a in range(self.dim):
                self.axes[a].release(int(pl.axis_off[a]), pl.axis_len[a])


def ctypes_ref(P):
    import ctypes
    return ctypes.byref(P)


class RoundPack(Pack):
    """A pack over arena storage listing a set of resident devices: the
    per-instance tables are built for the set, the node arrays are the
    arena's (n_nodes = arena capacity)."""

    autotune = False     # resident devices keep their placement's tiles

    def __init__(self, arena, sessions):
        sessions = sorted(sessions, key=lambda s: s.pl.off)
        self.sessions = sessions
        self._init_common([s.setup for s in sessions], arena.device)
        if len(sessions) > arena.max_inst:
            raise ValueError("more instances than the arena's workspace holds")
        self.arena = arena
        self.t = dict(arena.t)
        self.N = arena.cap
        dim = self.dim
        self._set_tables(instance_tables(
            self.setups, dim, [s.pl.off for s in sessions],
            np.stack([s.pl.axis_off for s in sessions]), [s.pl.tiles for s in sessions],
            tile_z=TILE_Z if dim == 3 else 1))
        self.psi, self.n, self.p = arena.psi, arena.n, arena.p
        self.F, self.J, self.du, self.work = arena.F, arena.J, arena.du, arena.work
        self._prev = arena.prev
        self.active = self.torch.ones(len(sessions), dtype=self.torch.uint8,
                                      device=self.device)
        self._contact_tables([s.pl.ctab for s in sessions])
        self._build_gate_map(cached=[(s.pl.gm, s.pl.gnodes) for s in sessions])

    def refresh_bcs(self):       # the arena holds the BC arrays already
        raise NotImplementedError


def own_setup(setup):
    """A copy of a Setup whose contacts and gates are its own objects (the
    coefficient arrays stay shared, read-only): the bias a session applies
    lives on its BC objects, so two sessions built from one Setup must not
    share them."""
    own = copy.copy(setup)
    own.bcs = {name: copy.copy(b) for name, b in setup.bcs.items()}
    return own


class Session:
    """A device resident (or to be resident) in an arena.  It owns its BC
    objects (own_setup), so requests that share a Setup keep their biases."""

    def __init__(self, key, setup):
        self.key = key
        self.setup = own_setup(setup)
        self.pl = None
        self.bias_prev = self.bias_cur = None
        self.need_eq = True
        self.fresh_guess = False
        self.busy = False


class Request:
    """Bias points to solve on one device.  points: list of {name: V};
    report: which points' currents are returned; contact: the terminal whose
    current is reported."""

    def __init__(self, key, setup, points, contact, report=None, arrival=None,
                 from_equilibrium=True, return_state=False):
        self.key = key
        self.from_equilibrium = from_equilibrium
        self.return_state = return_state
        self.state = None
        self.setup = setup
        self.points = list(points)
        self.report = list(report) if report is not None else [True] * len(self.points)
        self.contact = contact
        self.arrival = time.perf_counter() if arrival is None else arrival
        self.next = 0
        self.currents = []
        self.converged = []
        self.newton = []
        self.finished = None
        self.error = None
        self.done = threading.Event()

    @property
    def latency(self):
        return None if self.finished is None else self.finished - self.arrival

    @property
    def reported_points(self):
        return sum(1 for r in self.report if r)


class Worker(threading.Thread):
    """Serves the requests of one dimension from one arena, on its own CUDA
    stream, round after round."""

    def __init__(self, dim, budget_bytes, opts, device="cuda", max_inst=4096,
                 max_round_nodes=None):
        super().__init__(daemon=True)
        import torch
        self.torch = torch
        self.dim = dim
        self.opts = opts
        dev = torch.device(device)
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.arena = Arena(dim, budget_bytes, device, max_inst)
        self.max_round_nodes = max_round_nodes or self.arena.cap
        self.stream = torch.cuda.Stream(device=self.device)
        self.queue = collections.deque()
        self.cv = threading.Condition()
        self.sessions = collections.OrderedDict()      # key -> Session, LRU first
        self.active = []                               # requests in flight
        self.running = True
        self.aborting = False
        self.rounds = 0
        self.round_log = []
        self.h2d_bytes = 0
        self.d2h_bytes = 0
        self.error = None

    # ---- client side
    def submit(self, req):
        with self.cv:
            self.queue.append(req)
            self.cv.notify()

    def stop(self, abort=False):
        """Stop after the queue and the requests in flight are served; with
        abort, drop the queue and stop after the current round (requests
        still in flight are marked cancelled)."""
        with self.cv:
            self.running = False
            self.aborting = abort
            if abort:
                for r in self.queue:
                    r.error = "cancelled"
                self.queue.clear()
            self.cv.notify()

    def idle(self):
        with self.cv:
            return not self.queue and not self.active

    # ---- scheduling
    def _session_for(self, req):
        s = self.sessions.get(req.key)
        if s is None:
            s = Session(req.key, req.setup)
            self.sessions[req.key] = s
        else:
            self.sessions.move_to_end(req.key)   # same key: the same device
        return s

    def _evict_for(self, n):
        """Release idle resident devices, least recently used first, until a
        range of n nodes is free; True when it is."""
        ar = self.arena
        for key in list(self.sessions):
            if ar.nodes.largest() >= n:
                break
            s = self.sessions[key]
            if s.busy or s.pl is None:
                continue
            ar.release(s.pl)
            s.pl = None
            del self.sessions[key]
        return ar.nodes.largest() >= n

    def _admit(self):
        """Move queued requests in flight while the arena has room and the
        round stays within max_round_nodes; first fit over the queue."""
        admitted = []
        nodes = sum(r._session.setup.N for r in self.active)
        with self.cv:
            pending = list(self.queue)
        keep = []
        for req in pending:
            s = self.sessions.get(req.key)
            n = req.setup.N
            if (s is not None and s.busy) or (nodes > 0 and nodes + n > self.max_round_nodes) \
                    or len(self.active) + len(admitted) >= self.arena.max_inst:
                keep.append(req)
                continue
            s = self._session_for(req)
            if s.pl is None:
                if n > self.arena.cap:
                    req.error = "device larger than the arena"
                    req.finished = time.perf_counter()
                    req.done.set()
                    continue
                if not self._evict_for(n):
                    keep.append(req)
                    continue
                s.pl = self.arena.place(s.setup)
                if s.pl is None:
                    keep.append(req)
                    continue
                self.h2d_bytes += s.pl.h2d_bytes
                s.need_eq = True
                s.fresh_guess = True
            elif req.from_equilibrium:
                s.need_eq = True
                s.fresh_guess = False
            s.busy = True
            req._session = s
            nodes += n
            admitted.append(req)
        with self.cv:
            taken = set(id(r) for r in pending) - set(id(r) for r in keep)
            self.queue = collections.deque(r for r in self.queue if id(r) not in taken)
        return admitted

    def run_round(self):
        """Admit, bring new devices to equilibrium, then solve the next bias
        point of every request in flight in one batched Newton solve."""
        admitted = self._admit()
        self.active.extend(admitted)
        if not self.active:
            return False
        t0 = time.perf_counter()
        new = [r._session for r in self.active if r._session.need_eq]
        if new:
            for s in new:
                if not s.fresh_guess:         # resident device: restart from the guess
                    g = self.torch.from_numpy(s.setup.bulk_guess().ravel())
                    self.arena.psi[s.pl.off:s.pl.off + s.pl.n].copy_(g)
                    self.h2d_bytes += g.numel() * 8
                s.fresh_guess = False
            RoundPack(self.arena, new).equilibrium(self.opts)
            self.stream.synchronize()
            for s in new:
                s.need_eq = False
                s.bias_prev, s.bias_cur = None, np.zeros(len(s.setup.bcs))
        t_eq = time.perf_counter() - t0
        sessions = [r._session for r in self.active]
        for r in self.active:
            for name, V in r.points[r.next].items():
                b = r._session.setup.bcs[name]
                if b.kind == "contact":
                    b.V = float(V)
                else:
                    b.Vg = float(V)
        rp = RoundPack(self.arena, sessions)
        rp.set_bias()
        self.h2d_bytes += rp.last_h2d_bytes
        opts = self.opts
        use_pred = getattr(opts, "predictor", "none") == "secant"
        newb = [bias_vector(s.setup) for s in rp.sessions]
        ratios = [secant_ratio(s.bias_prev, s.bias_cur, b) if use_pred else 0.0
                  for s, b in zip(rp.sessions, newb)]
        if use_pred:
            rp.predict(ratios)
        rp.stamp_contacts()
        res = rp.newton(opts)
        retry = [i for i, r in enumerate(ratios) if r != 0.0 and not res[i]["converged"]]
        if retry:      # predicted starts that failed: again from the previous state
            rp.restore_prev(retry)
            mask = np.zeros(len(rp.sessions), dtype=bool)
            mask[retry] = True
            rp.stamp_contacts(mask)
            res2 = rp.newton(opts, active=mask)
            for i in retry:
                res2[i]["iters"] += res[i]["iters"]
                res2[i]["krylov_iters"] += res[i]["krylov_iters"]
                res[i] = res2[i]
        for s, b, rr in zip(rp.sessions, newb, res):
            s.bias_prev = s.bias_cur if use_pred else None
            s.bias_cur = b if rr["converged"] else None
        by_session = {id(s): (i, res[i]) for i, s in enumerate(rp.sessions)}
        outs = []
        for r in self.active:
            i, rr = by_session[id(r._session)]
            if r.report[r.next]:
                outs.append((r, i, rr))
            else:
                r.newton.append(rr)
        if outs:
            for k, (r, i, _) in enumerate(outs):
                rp.contact_current(i, r.contact, out_slot=k)
            cur = rp.cur_out[:len(outs)].cpu().numpy()
            self.d2h_bytes += cur.nbytes
            exp = 1 if self.dim == 2 else 2
            for (r, i, rr), c in zip(outs, cur):
                s = r._session.setup
                r.currents.append(float(c) * s.J0 * s.LD ** exp)
                r.converged.append(bool(rr["converged"]))
                r.newton.append(rr)
        now = time.perf_counter()
        still = []
        for r in self.active:
            r.next += 1
            if r.next >= len(r.points):
                if r.return_state:
                    pl = r._session.pl
                    r.state = tuple(a[pl.off:pl.off + pl.n].cpu().numpy().reshape(
                        r._session.setup.shape) for a in (self.arena.psi, self.arena.n,
                                                          self.arena.p))
                r.finished = now
                r._session.busy = False
                r.done.set()
            else:
                still.append(r)
        self.active = still
        self.rounds += 1
        self.round_log.append((t0, now, len(sessions), len(new),
                               max(rr["iters"] for rr in res),
                               sum(1 for rr in res if not rr["converged"]),
                               sum(s_.setup.N for s_ in sessions), t_eq,
                               max(rr["krylov_iters"] for rr in res)))
        return True

    def run(self):
        torch = self.torch
        try:
            torch.cuda.set_device(self.device)
            with torch.cuda.stream(self.stream):
                while True:
                    with self.cv:
                        while self.running and not self.queue and not self.active:
                            self.cv.wait(0.05)
                        if not self.running and not self.active and not self.queue:
                            break
                        if self.aborting:
                            for r in self.active:
                                r.error = "cancelled"
                                r._session.busy = False
                            self.active = []
                            break
                    self.run_round()
                self.stream.synchronize()
        except Exception as exc:     # fail what is in flight and queued, stop
            self.error = exc
            with self.cv:
                failed = self.active + list(self.queue)
                self.queue.clear()
            for r in failed:
                r.error = repr(exc)
                r.finished = time.perf_counter()
                r.done.set()
            self.active = []


# Default cap of the nodes one round solves.  A 2D round's time is set by its
# members' Newton steps under ILU(0) sweeps (one dependent level per
# anti-diagonal, up to 767 for 512 x 256) and, in a round that admits many
# devices, by their equilibrium solves.  Measured at 200 req/s: rounds of
# ~160 devices (6.4M nodes) took 7 s at the median, rounds of ~300-700
# devices (13M) 29-70 s -- and a single-bias request needs 4 rounds, a sweep
# 13-43, so long rounds leave every request unfinished in a minute-long
# window.  8M 2D nodes keeps rounds short; 3D rounds (block Jacobi, no
# sweeps) scale with their nodes and stay at 4M.
ROUND_NODES = {2: 8_000_000, 3: 4_000_000}


class Server:
    """Continuous-batching service: one Worker (arena, stream, thread) per
    dimension.  budget: HBM bytes per dimension."""

    def __init__(self, budget=None, opts=None, device="cuda", max_inst=4096,
                 max_round_nodes=None):
        budget = budget or {2: 8 << 30, 3: 8 << 30}
        self.opts = opts or NewtonOptions(precision="mixed")
        caps = dict(ROUND_NODES, **(max_round_nodes or {}))
        self.workers = {d: Worker(d, b, self.opts, device, max_inst, caps.get(d))
                        for d, b in budget.items()}

    def start(self):
        for w in self.workers.values():
            w.start()
        return self

    def submit(self, req):
        self.workers[req.setup.dim].submit(req)
        return req

    def stop(self, abort=False):
        for w in self.workers.values():
            w.stop(abort)
        for w in self.workers.values():
            w.join()

    def wait_idle(self, timeout=None):
        t_end = None if timeout is None else time.perf_counter() + timeout
        while not all(w.idle() for w in self.workers.values()):
            for w in self.workers.values():
                if w.error is not None:
                    raise RuntimeError(f"{w.dim}D worker failed") from w.error
            if t_end is not None and time.perf_counter() > t_end:
                return False
            time.sleep(0.002)
        for w in self.workers.values():
            if w.error is not None:
                raise RuntimeError(f"{w.dim}D worker failed") from w.error
        return True
