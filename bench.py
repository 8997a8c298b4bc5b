#!/usr/bin/env python
"""Converged bias points per second of the drift-diffusion solve on B200.

Workload (default): the 3D n-channel tri-gate on a 160 x 96 x 64 tensor mesh
(983,040 nodes, 2,949,120 unknowns): p-body 1e18, Gaussian S/D implants of
peak 1e20 cm^-3 (sigma 10 nm), 40 nm gate, 1 nm oxide Robin gates on three
faces; Id-Vg sweep Vg = 0..1.0 V in 21 steps at Vd = 0.05 V and at 0.7 V,
each sweep warm-started from equilibrium.  Synthetic device (no dataset).

One step = one Vg on BOTH Vd branches: two warm-started bias points, solved
as one packed 2-instance batch by the chosen path (the plain path solves the
two branch devices one after another), + the terminal currents.  The warm-up
steps walk the start of the schedule, then the schedule restarts, so K timed
steps cover Vg = 0 .. 0.05 (K-1) V on both branches, equilibrium included.
A point counts only when Newton converged (update < 1e-8 plus the polishing
steps) and its current is within 1e-6 of the reference current: the plain
FP64 path's state at that point, solved on untimed to the oracle fixtures'
setting (update test 1e-12, Krylov at 1e-10 in relative unknowns).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--workload trigate3d|diode2d|pin3d|mosfet2d_batch|serve]
                  [--method fp64|full|plain|mixed|fp32op|rb_bj] [--no-fused]
                  [--small] [--kernels]

N > 1: one process per GPU under torchrun, each an independent replica of the
sweep (the path does not shard: replicas only); value = all ranks' points /
max-over-ranks time.  --impl reference: the oracle's CPU implementation of
the same path on the host cores (rank 0 only).
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "converged bias pts/s at <=1e-6 rel current err, chosen vs plain GPU; p50/p99"
UNIT = "bias_pts/s"

# Algorithmic bytes per node (one launch touches every node once):
#  block SpMV (scaled, 3D): J 39 doubles + x 3 + y 3             = 360 B
#  coupled SG assembly (3D): 16 doubles in (psi,n,p,C,nie,tau_n,tau_p,
#     an/ap/dl x 3 axes) + bcflag byte + 42 doubles out (F 3, J 39) = 465 B
BYTES_SPMV = {2: (29 + 3 + 3) * 8, 3: (39 + 3 + 3) * 8}
BYTES_ASM = {2: (13 + 32) * 8 + 1, 3: (16 + 42) * 8 + 1}
#  one BiCGStab iteration in the solver (node-block layout, FP64), bytes per
#  node of the five kernels: k_bi_p 96 (r, v, p in; p out), k_bi_v and k_bi_t
#  one SpMV each (J + x in, y out), k_bi_s 72, k_bi_x 168
BYTES_ITER = {d: 96 + 2 * BYTES_SPMV[d] + 72 + 168 for d in (2, 3)}
#  one BiCGStab iteration on the red-black Schur complement, bytes per node of
#  the original pack (a black slot per two nodes): the vector kernels on the
#  black half (96 + 72 + 168) / 2; two red passes (red rows of J, black x in,
#  E x out: (8 NE + 48) / 2 each); the black passes (black rows of J, E x, one
#  vector in, product out, plus rh for v: (8 NE + 96) / 2 and (8 NE + 72) / 2)
#  = 300 + 16 NE: 924 in 3D, 764 in 2D
BYTES_ITER_RB = {d: 300 + 16 * (29 if d == 2 else 39) for d in (2, 3)}

# Newton iterations / BiCGStab iterations per bias point of the plain FP64
# path on this workload, from its own bench runs; used only to scale the
# CPU oracle's measured per-iteration costs to a bias point.
TRIGATE_ITERS = {"newton_per_point": 6.0, "krylov_per_newton": 1078.0}


# The Newton/Krylov methods the bench can time.  "plain" is the reference's
# iterative semantics on the GPU kernels: every Newton step's BiCGStab solved
# to the fixed rtol 1e-10 on (dpsi, dn, dp) with node-block Jacobi.
METHODS = {
    "plain": dict(precision="fp64", forcing="fixed", krylov_unknowns="absolute",
                  predictor="none", krylov_system="full"),
    "fp64": dict(precision="fp64", forcing="adaptive", krylov_unknowns="relative",
                 predictor="secant", krylov_system="red_black"),
    "full": dict(precision="fp64", forcing="adaptive", krylov_unknowns="relative",
                 predictor="secant", krylov_system="full"),
    "mixed": dict(precision="mixed", forcing="adaptive", krylov_unknowns="relative",
                  predictor="secant"),
    "fp32op": dict(precision="fp32_operator", forcing="adaptive", krylov_unknowns="relative",
                   predictor="secant"),
    "rb_bj": dict(precision="fp64", forcing="adaptive", krylov_unknowns="relative",
                  predictor="secant", krylov_system="red_black", precond="block_jacobi"),
}
METHOD_DESC = {
    "plain": "plain FP64: fused SG assembly, node-block-Jacobi BiCGStab to rtol 1e-10 on "
             "(dpsi, dn, dp) every Newton step, damped Newton",
    "fp64": "FP64 inexact Newton: fused SG assembly, BiCGStab on the red-black Schur "
            "complement of the block-scaled system (red nodes eliminated exactly; the full "
            "system's stopping test) in relative unknowns (dpsi, dn/n, dp/p) solved to 1e-3 "
            "every Newton step, two polishing steps (1e-6, then 1e-3), secant predictor "
            "along the sweep",
    "full": "as 'fp64', with the BiCGStab on the whole block-scaled system",
    "fp32op": "FP64 inexact Newton as 'fp64', but the BiCGStab of the Newton steps before the "
              "update test reads an FP32 copy of the block-scaled Jacobian (FP64 vectors, dots "
              "and polishing steps)",
    "rb_bj": "as 'fp64', with node-block Jacobi for every instance (2D batches included, "
             "which otherwise take ILU(0))",
    "mixed": "mixed precision inexact Newton: FP64 assembly, residual, Newton update and "
             "convergence test; FP32 block-scaled BiCGStab inside FP64 iterative refinement, "
             "relative unknowns, adaptive forcing, secant predictor; per-instance FP64 "
             "fallback when an FP32-solved step is rejected",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="trigate3d",
                    choices=["trigate3d", "diode2d", "pin3d", "mosfet2d_batch", "serve"])
    ap.add_argument("--duration", type=float, default=60.0,
                    help="serve: seconds of Poisson arrivals")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: mean requests/s")
    ap.add_argument("--budget-gb", type=float, default=160.0,
                    help="serve: HBM budget of the arenas (GB)")
    ap.add_argument("--drain", type=float, default=120.0,
                    help="serve: seconds to finish in-flight work after the arrivals end")
    ap.add_argument("--plain-seconds", type=float, default=45.0,
                    help="serve: time cap of the sequential plain FP64 run")
    ap.add_argument("--batch", type=int, default=512,
                    help="mosfet2d_batch: instances in the batch")
    ap.add_argument("--plain-sample", type=int, default=16,
                    help="mosfet2d_batch: instances of the sequential plain run")
    ap.add_argument("--small", action="store_true", help="down-scaled mesh (testing)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--method", default="fp64", choices=list(METHODS),
                    help="the timed (chosen) path; the plain FP64 path is always run "
                         "beside it on the same points for the current check")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--asm-stage", type=int, default=0, choices=(0, 1),
                    help="--kernels: the 3D assembly's plane staging (pack asm_stage)")
    ap.add_argument("--no-fused", action="store_true",
                    help="solve single-instance packs one launch per Krylov step (the "
                         "red-black Schur loop for FP64 block-Jacobi solves) instead of "
                         "the one-launch BiCGStab")
    ap.add_argument("--kernels", action="store_true",
                    help="profiling mode: assembly, block-Jacobi set-up and 20 BiCGStab "
                         "iterations on the full-size workload at its bulk-guess state")
    return ap.parse_args()


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def load_traffic(name):
    """Bytes per launch of a kernel from its committed ncu summary
    (profiles/<name>.md, line 'traffic_bytes_per_launch: <int>'), else None."""
    p = os.path.join(ROOT, "profiles", name + ".md")
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(float(line.split(":")[1]))
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def build_workload(name, small, dev_cls_2d, dev_cls_3d):
    """(lanes, steps, description, contact).  A lane is one device marching
    through its own bias points; a step gives every lane its next point:
    steps[q] = ([volts of lane 0, lane 1, ...], starts_from_equilibrium)."""
    from tcad_b200 import workloads as W
    if name == "pin3d":
        dims = (64, 32, 16) if small else (256, 256, 128)
        lanes = [W.pin3d(dev_cls_3d, *dims)]
        steps = [([{"anode": v}], i == 0) for i, v in enumerate(W.PIN_SWEEP)]
        desc = (f"pin3d {dims[0]}x{dims[1]}x{dims[2]} ({int(np.prod(dims)):,} nodes) p+ 1e19 / "
                "i 1e14 / n+ 1e19, 20 nm erfc transitions, SRH + Auger, forward 0..0.9 V "
                "step 0.1")
        return lanes, steps, desc, "anode"
    if name == "diode2d":
        nx, ny = (41, 11) if small else (201, 101)
        lanes = [W.diode2d(dev_cls_2d, nx, ny)]
        steps = [([{"anode": v}], i == 0) for i, v in enumerate(W.DIODE_SWEEP)]
        desc = f"diode2d {nx}x{ny} ({nx * ny} nodes) 0..0.7 V step 0.05"
        return lanes, steps, desc, "anode"
    dims = (40, 24, 16) if small else (160, 96, 64)
    lanes = [W.trigate3d(dev_cls_3d, *dims) for _ in W.TRIGATE_VD]
    steps = [([W.trigate_bias(vd, vg) for vd in W.TRIGATE_VD], q == 0)
             for q, vg in enumerate(W.TRIGATE_VG)]
    desc = (f"trigate3d {dims[0]}x{dims[1]}x{dims[2]} ({np.prod(dims):,} nodes) Id-Vg "
            "Vg 0..1.0 V step 0.05 at Vd 0.05 V and 0.7 V; one step = one Vg on both "
            "Vd branches (2 bias points)")
    return lanes, steps, desc, "drain"


class SweepRunner:
    """The workload's lanes marching through the bias schedule with one Newton
    method.  batched: all lanes in ONE packed DeviceBatch (every launch covers
    both Vd branches, per-instance Newton/Krylov masks); otherwise the lanes'
    devices are solved one after another, as the reference would."""

    def __init__(self, args, method, dev_classes, batched):
        import tcad_b200 as tb
        from tcad_b200.batch import DeviceBatch
        self.args = args
        self.lanes, self.steps, self.desc, self.contact = build_workload(
            args.workload, args.small, *dev_classes)
        self.opts = tb.NewtonOptions(verbose=bool(args.verbose), **METHODS[method])
        self.method = method
        self.batch = DeviceBatch(self.lanes) if batched and len(self.lanes) > 1 else None
        self.q = 0
        self.log = []
        self.N = sum(d.N for d in self.lanes)

    def restart(self):
        """Back to the first step (the next step starts from equilibrium)."""
        self.q = 0

    def step(self):
        """Solve every lane's next point; returns (currents, converged flags,
        h2d bytes, d2h bytes)."""
        volts, first = self.steps[self.q % len(self.steps)]
        self.q += 1
        if self.batch is not None:
            b = self.batch
            if first:
                b.solve_equilibrium(self.opts)
            res = b.solve_bias(volts, self.opts)
            I = list(b.terminal_currents(self.contact))
            conv = [r["converged"] for r in res]
            h2d = b.pack.last_h2d_bytes
        else:
            I, conv, res, h2d = [], [], [], 0
            for dev, v in zip(self.lanes, volts):
                if first:
                    dev.solve_equilibrium(self.opts)
                dev.solve_bias(v, self.opts)
                I.append(dev.terminal_current(self.contact))
                conv.append(bool(dev.last_converged))
                res.append(dev.last_newton)
                h2d += dev.pack.last_h2d_bytes   # contact targets + gate-node values
        for lane, (r, i, v) in enumerate(zip(res, I, volts)):
            self.log.append(dict(r, first=first, I=i, lane=lane))
            if self.args.verbose:
                sys.stderr.write(f"  [{self.method}] step {self.q:3d} lane {lane} {v} "
                                 f"first={first} conv={r['converged']} newton={r['iters']} "
                                 f"krylov={r['krylov_iters']} relres={r['relres']:.1e} "
                                 f"I={i:.9e}\n")
                sys.stderr.flush()
        return I, conv, h2d, 8 * len(I)

    def read_fields(self):
        """Host read of every lane's potential field (the e2e result copy);
        returns the bytes read."""
        if self.batch is not None:
            _ = self.batch.pack.psi.cpu()
        else:
            for dev in self.lanes:
                _ = dev.psi
        return 8 * self.N

    def reference_currents(self):
        """The currents of the tightly converged solutions at the last step:
        each lane's state solved on, untimed, with relative Krylov unknowns at
        1e-10 every step and the update test at 1e-12 (plus the polishing
        step) -- the fixtures' oracle-quality setting: at the stock 1e-8 the
        update test saturates at the 1e-10 density floor, so sub-floor
        minority densities, and the currents that depend on them, are only
        loosely converged.  States are put back afterwards, so the runner's
        own march is unchanged.  (Sequential lanes only.)"""
        import tcad_b200 as tb
        volts, _ = self.steps[(self.q - 1) % len(self.steps)]
        ref = tb.NewtonOptions(precision="fp64", forcing="adaptive",
                               krylov_unknowns="relative", predictor="none",
                               eta_max=1e-10, eta_min=1e-10, tol_update=1e-12,
                               krylov_system="full")
        out = []
        for dev, v in zip(self.lanes, volts):
            keep = [t.clone() for t in (dev.pack.psi, dev.pack.n, dev.pack.p)]
            attrs = {k: getattr(dev, k) for k in ("_bias_prev", "_bias_cur", "last_newton",
                                                  "last_converged")}
            dev.solve_bias(v, ref)
            out.append(dev.terminal_current(self.contact) if dev.last_converged
                       else float("nan"))
            for t, k in zip((dev.pack.psi, dev.pack.n, dev.pack.p), keep):
                t.copy_(k)
            for k, val in attrs.items():
                setattr(dev, k, val)
            dev._host.clear()
        return out

    def release(self):
        self.lanes = self.batch = None


def timed_steps(torch, runner, steps, e2e, ref_currents=None):
    """Per-step device latency (CUDA events on the launching stream) and, with
    e2e, the latency including the host read of the potential fields.  With
    ref_currents (a list), each point's tightly converged reference current
    is appended to it, untimed."""
    lat, lat_e2e, conv, h2d, d2h = [], [], 0, 0, 0
    for _ in range(steps):
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record()
        I, ok, hb, db = runner.step()
        b.record()
        if e2e:
            db += runner.read_fields()
        c.record()
        torch.cuda.synchronize()
        lat.append(a.elapsed_time(b))
        lat_e2e.append(a.elapsed_time(c))
        conv += int(sum(ok))
        h2d += hb
        d2h += db
        if ref_currents is not None:
            ref_currents.extend(runner.reference_currents())
    return lat, lat_e2e, conv, h2d, d2h


def reduce_over_ranks(dist, device, t_dev, t_e2e, ok_pts):
    """Whole-job figures of independent replicas: the slowest rank's device
    and end-to-end times, and the points all ranks counted.  Every rank calls
    it once, at the same place (two all-reduces, MAX then SUM)."""
    import torch
    tt = torch.tensor([t_dev, t_e2e], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    cc = torch.tensor([ok_pts], device=device, dtype=torch.float64)
    dist.all_reduce(cc, op=dist.ReduceOp.SUM)
    return float(tt[0]), float(tt[1]), int(cc.item())


def run_ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import tcad_b200 as tb
    from tcad_b200 import _lib
    lib = _lib.load()
    classes = (tb.Device2D, tb.Device3D)
    chosen = SweepRunner(args, args.method, classes, batched=True)
    dev = chosen.lanes[0]
    dim, N = dev.dim, dev.N
    ppstep = len(chosen.lanes)          # bias points per step

    for _ in range(args.warmup):
        chosen.step()
    chosen.restart()                    # the timed steps walk the schedule from its start
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    L0 = lib.tcad_launch_count()
    n_warm_log = len(chosen.log)
    with Clocks(local) as clk:
        t_wall = time.perf_counter()
        lat, lat_e2e, conv, h2d_tot, d2h_tot = timed_steps(torch, chosen, args.steps, True)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t_wall
    launches = lib.tcad_launch_count() - L0
    t_dev = sum(lat) / 1e3
    t_e2e = sum(lat_e2e) / 1e3
    pts_chosen = chosen.log[n_warm_log:]

    # the plain FP64 path on the same points, its lanes one after another:
    # its throughput, and the reference currents for the chosen path's 1e-6
    # check
    plain_lat = None
    if args.method != "plain":
        plain = SweepRunner(args, "plain", classes, batched=False)
        for _ in range(args.warmup):
            plain.step()
        plain.restart()
        n0 = len(plain.log)
        I_ref = []
        plain_lat, _, plain_conv, _, _ = timed_steps(torch, plain, args.steps, False, I_ref)
        pts_plain = plain.log[n0:]
        rel = lambda a, b: abs(a - b) / max(abs(b), 1e-300)  # noqa: E731
        errs = [rel(c["I"], p["I"]) for c, p in zip(pts_chosen, pts_plain)]
        errs_ref = [rel(c["I"], r) for c, r in zip(pts_chosen, I_ref)]
        errs_plain_ref = [rel(p["I"], r) for p, r in zip(pts_plain, I_ref)]
        plain_counts = ([r["iters"] for r in pts_plain], [r["krylov_iters"] for r in pts_plain])
        ok_pts = sum(1 for c, e in zip(pts_chosen, errs_ref) if c["converged"] and e <= 1e-6)
        plain.release()
        del plain
    else:
        errs = [0.0] * len(pts_chosen)
        errs_ref = errs_plain_ref = None
        ok_pts = conv
        plain_conv = conv
        plain_counts = ([r["iters"] for r in pts_chosen], [r["krylov_iters"] for r in pts_chosen])

    if world > 1:
        t_dev, t_e2e, ok_all = reduce_over_ranks(dist, "cuda", t_dev, t_e2e, ok_pts)
    else:
        ok_all = ok_pts

    # ---- live roofline of the dominant kernel (block SpMV on the last J) and
    # of the assembly, CUDA events on the launching stream
    pk = chosen.batch.pack if chosen.batch is not None else dev.pack
    NN = pk.N                            # nodes of the timed pack (every lane)
    sp = _lib.stream_ptr()
    y = torch.empty_like(pk.du)
    x = torch.randn(3 * pk.N, dtype=torch.float64, device=pk.device)

    def time_kernel(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    pk.assemble(_lib.MODE_ELIMINATE)
    st = torch.zeros(max(1, len(pk.setups)), dtype=torch.int32, device=pk.device)
    lib.tcad_block_jacobi_setup(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F), _lib.ptr(st), sp)
    t_spmv = time_kernel(lambda: lib.tcad_block_spmv(pk.pref, _lib.ptr(pk.J), _lib.ptr(x),
                                                     _lib.ptr(y), sp), 50)
    Fa = torch.empty_like(pk.F)
    Ja = torch.empty_like(pk.J)
    t_asm = time_kernel(lambda: lib.tcad_sg_assemble(pk.pref, _lib.ptr(pk.psi), _lib.ptr(pk.n),
                                                     _lib.ptr(pk.p), _lib.ptr(Fa), _lib.ptr(Ja),
                                                     _lib.MODE_ELIMINATE, sp), 20)
    # one whole BiCGStab iteration inside the solver (five fused kernels),
    # timed as a fixed-count solve that cannot converge
    ni = pk.P.n_inst
    kit, kst, krr = (ctypes.c_int32 * ni)(), (ctypes.c_int32 * ni)(), (ctypes.c_double * ni)()
    xk = torch.zeros_like(pk.du)
    KIT = 200

    rb = METHODS[args.method].get("krylov_system") == "red_black"
    kmethod = 2 if rb else 0
    bytes_iter = (BYTES_ITER_RB if rb else BYTES_ITER)[dim]

    def krylov_fixed():
        lib.tcad_block_krylov(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F), _lib.ptr(xk), kmethod,
                              1e-300, KIT, 0, _lib.ptr(pk.work), pk.work.numel(), kit, kst,
                              krr, sp)
    t_kry = time_kernel(krylov_fixed, 2)
    it_done = max(int(kit[i]) for i in range(ni))
    t_iter = t_kry / max(it_done, 1)
    peak, peak_kind = load_peaks()
    ach_spmv = BYTES_SPMV[dim] * NN / t_spmv / 1e9
    ach_asm = BYTES_ASM[dim] * NN / t_asm / 1e9
    ach_iter = bytes_iter * NN / t_iter / 1e9
    lane_traffic = load_traffic(("rb_iteration" if rb else "bicgstab_iteration")
                                + f"_{args.workload}")
    iter_traffic = (lane_traffic * NN / chosen.lanes[0].N
                    if lane_traffic is not None else None)

    res = {}
    if rank == 0:
        nn = [r["iters"] for r in pts_chosen]
        kk = [r["krylov_iters"] for r in pts_chosen]
        value = ok_all / t_dev
        method_desc = METHOD_DESC[args.method]
        res = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_dev / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"mixed": "f64 (FP32 inner Krylov)",
                      "fp32op": "f64 (FP32 operator copy)"}.get(args.method, "f64"),
            "data": "synthetic device (analytic doping profiles, explicit mesh)",
            "config": {"workload": chosen.desc, "method": method_desc,
                       "single_launch_bicgstab": not args.no_fused,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (J alone is "
                             f"{8 * _lib.NE[dim] * N / 1e6:.0f} MB)"},
            "p50_ms": statistics.median(lat), "p99_ms": float(np.percentile(lat, 99)),
            "converged_points": conv, "points_within_1e-6_of_reference": ok_pts,
            "points": args.steps * world * ppstep, "points_per_step": ppstep,
            "current_reference": "each timed point's plain FP64 state solved on, untimed, "
                                 "to the oracle fixtures' setting (relative unknowns at "
                                 "1e-10, update test 1e-12, polishing step)",
            "max_rel_current_err_vs_reference": float(np.max(errs_ref)) if errs_ref else None,
            "max_rel_current_err_plain_vs_reference":
                float(np.max(errs_plain_ref)) if errs_plain_ref else None,
            "max_rel_current_err_vs_plain_fp64": float(max(errs)) if errs else None,
            "fp64_fallback_points": sum(1 for r in pts_chosen if r.get("fp64_from", -1) >= 0),
            "newton_iters_mean": float(np.mean(nn)), "krylov_iters_mean": float(np.mean(kk)),
            "e2e": {"value": ok_all / t_e2e, "unit": UNIT,
                    "h2d_bytes_per_step": int(h2d_tot / args.steps),
                    "d2h_bytes_per_step": int(d2h_tot / args.steps),
                    "p50_ms": statistics.median(lat_e2e),
                    "p99_ms": float(np.percentile(lat_e2e, 99))},
            # the dominant work: one Krylov iteration (96 % of a bias point),
            # timed as a fixed-count solve on the timed pack; traffic from the
            # committed ncu summary of one iteration on one lane, scaled by the
            # pack's node count
            "roofline": {
                "kernel": ("k_bi_p + k_rb_red + k_rb_v + k_bi_s + k_rb_red + k_rb_t + k_bi_x "
                           "(one red-black Schur BiCGStab iteration, all lanes)" if rb else
                           "k_bi_p + k_bi_v + k_bi_s + k_bi_t + k_bi_x (one BiCGStab "
                           "iteration, all lanes)"),
                "bound": "hbm", "achieved": ach_iter, "peak": peak, "unit": "GB/s",
                "frac": ach_iter / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "bytes_per_launch": bytes_iter * NN, "launch_ms": t_iter * 1e3,
                "iterations_timed": it_done,
                "traffic": iter_traffic},
            "roofline_spmv": {"kernel": "k_spmv (node-block SpMV of the whole scaled system, "
                                        "FP64)",
                              "bound": "hbm", "achieved": ach_spmv, "peak": peak,
                              "unit": "GB/s", "frac": ach_spmv / peak,
                              "bytes_per_launch": BYTES_SPMV[dim] * NN,
                              "launch_ms": t_spmv * 1e3,
                              "traffic": load_traffic(f"spmv{dim}d_{args.workload}")},
            "roofline_assembly": {"kernel": "k_sg_assemble", "bound": "hbm",
                                  "achieved": ach_asm, "peak": peak, "unit": "GB/s",
                                  "frac": ach_asm / peak,
                                  "bytes_per_launch": BYTES_ASM[dim] * NN,
                                  "launch_ms": t_asm * 1e3,
                                  "traffic": load_traffic(f"assemble{dim}d_{args.workload}")},
            "gpu_launches": int(launches),
            "clocks": clk.summary(),
            "wall_s": wall,
        }
        if plain_lat is not None:
            res["plain_fp64_gpu"] = {
                "value": plain_conv / (sum(plain_lat) / 1e3), "unit": UNIT,
                "p50_ms": statistics.median(plain_lat),
                "p99_ms": float(np.percentile(plain_lat, 99)),
                "converged_points": plain_conv}
            res["chosen_over_plain"] = value / res["plain_fp64_gpu"]["value"]
        if world == 1 and not args.no_cpu_baseline:
            st0 = chosen.batch.state(0) if chosen.batch is not None else \
                (dev.psi, dev.n, dev.p)
            res["cpu_baseline"] = cpu_baseline(dev, st0, *plain_counts)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return res


# ---------------------------------------------------------------------------
# Batched 2D MOSFETs: one packed batch against sequential plain solves.
BATCH_RAMP = 4     # equal bias steps from equilibrium to each instance's (Vg, Vd)


def batch_devices(args, dev_cls, idx=None):
    from tcad_b200 import workloads as W
    params = W.mosfet_batch_params(args.batch)
    if args.small:
        params = [dict(q, nx=max(20, q["nx"] // 4), ny=max(12, q["ny"] // 4)) for q in params]
    idx = range(len(params)) if idx is None else idx
    out = []
    for i in idx:
        q = params[i]
        out.append((q, W.mosfet2d(dev_cls, nx=q["nx"], ny=q["ny"], Lg=q["Lg"], Na=q["Na"],
                                  Nsd_peak=q["Nsd_peak"])))
    return out


def run_batch(args):
    """512 seeded MOSFETs of uneven size, each at its own (Vg, Vd): a step is
    one packed solve of all of them (equilibrium, then BATCH_RAMP bias steps
    to the target) and the drain currents read back to the host.  The plain
    FP64 path solves an evenly spaced sample of the same instances one after
    another, the same way; its rate is points per second of that sample."""
    import torch
    import tcad_b200 as tb
    from tcad_b200 import _lib
    from tcad_b200 import workloads as W
    from tcad_b200.batch import DeviceBatch
    lib = _lib.load()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    t_build = time.perf_counter()
    built = batch_devices(args, tb.Device2D)
    params = [q for q, _ in built]
    batch = DeviceBatch([d for _, d in built])
    t_build = time.perf_counter() - t_build
    N = batch.pack.N
    opts = tb.NewtonOptions(verbose=bool(args.verbose), **METHODS[args.method])
    ramps = [W.ramp({"gate": q["Vg"], "drain": q["Vd"]}, BATCH_RAMP) for q in params]

    def step():
        h2d = 0
        batch.solve_equilibrium(opts)
        conv = np.zeros(batch.n, dtype=bool)
        iters = np.zeros(batch.n)
        kits = np.zeros(batch.n)
        for s in range(BATCH_RAMP):
            res = batch.solve_bias([r[s] for r in ramps], opts)
            h2d += batch.pack.last_h2d_bytes
            conv = np.array([r["converged"] for r in res])
            iters += [r["iters"] for r in res]
            kits += [r["krylov_iters"] for r in res]
        I = batch.terminal_currents("drain")   # device -> host
        return I, conv, h2d, 8 * batch.n, iters, kits

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    L0 = lib.tcad_launch_count()
    lat = []
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        for _ in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            I, conv, h2d, d2h, iters, kits = step()
            b.record()
            torch.cuda.synchronize()
            lat.append(a.elapsed_time(b))
    launches = lib.tcad_launch_count() - L0
    t_dev = sum(lat) / 1e3
    n_conv = int(conv.sum())

    # sequential plain solves of an evenly spaced sample, until the time cap
    sample = np.unique(np.linspace(0, batch.n - 1, min(args.plain_sample, batch.n)).astype(int))
    popts = tb.NewtonOptions(**METHODS["plain"])
    plain_lat, plain_I, plain_conv, plain_done = [], [], 0, []
    t_cap = time.perf_counter() + args.plain_seconds
    for j, (q, dev) in zip(sample, batch_devices(args, tb.Device2D, sample)):
        if time.perf_counter() > t_cap:
            break
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        dev.solve_equilibrium(popts)
        for volts in ramps[j]:
            dev.solve_bias(volts, popts)
        Ij = dev.terminal_current("drain")
        b.record()
        torch.cuda.synchronize()
        plain_lat.append(a.elapsed_time(b))
        plain_I.append(Ij)
        plain_done.append(int(j))
        plain_conv += int(dev.last_converged)
        dev._pack = None
    sample = plain_done
    errs = [abs(I[j] - Ij) / max(abs(Ij), 1e-300) for j, Ij in zip(sample, plain_I)
            if conv[j]]
    plain_rate = plain_conv / (sum(plain_lat) / 1e3) if plain_lat else None
    value = args.steps * n_conv / t_dev
    res = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t_dev / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (FP32 inner Krylov)" if args.method == "mixed" else "f64",
        "data": "synthetic devices (seeded MOSFET draws, analytic doping)",
        "config": {"workload": f"mosfet2d_batch: {batch.n} Device2D MOSFETs, nx~U[80,400], "
                               f"ny~U[40,200], seed 2026 ({N:,} nodes packed); each at its "
                               f"own (Vg, Vd) via {BATCH_RAMP} equal steps from equilibrium",
                   "method": METHOD_DESC[args.method] + "; one packed ragged batch, "
                             "per-instance convergence masks",
                   "parallelism": "single GPU",
                   "l2": f"inputs larger than L2 (J alone is {8 * 29 * N / 1e6:.0f} MB)"},
        "p50_ms": statistics.median(lat), "p99_ms": float(np.percentile(lat, 99)),
        "converged_points": n_conv, "points_per_step": batch.n,
        "newton_iters_mean_per_instance": float(iters.mean()),
        "krylov_iters_mean_per_instance": float(kits.mean()),
        "newton_iters_max_per_instance": float(iters.max()),
        "krylov_iters_max_per_instance": float(kits.max()),
        "step_ms": [float(x) for x in lat],
        "plain_fp64_gpu": {"value": plain_rate, "unit": UNIT,
                           "sample_instances": [int(j) for j in sample],
                           "p50_ms_per_instance": statistics.median(plain_lat)
                           if plain_lat else None,
                           "p99_ms_per_instance": float(np.percentile(plain_lat, 99))
                           if plain_lat else None,
                           "converged": plain_conv,
                           "note": "sequential Device2D solves (node-block-Jacobi BiCGStab at "
                                   "rtol 1e-10, the reference's iterative method) of an evenly "
                                   "spaced sample, stopped at the time cap"},
        "chosen_over_plain": value / plain_rate if plain_rate else None,
        "max_rel_current_err_vs_plain_fp64": float(max(errs)) if errs else None,
        "e2e": {"value": args.steps * n_conv / t_dev, "unit": UNIT,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "note": "the timed step already includes the bias uploads and the "
                        "current read-back"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
        "build_s": t_build,
    }
    return res


# ---------------------------------------------------------------------------
# Serving: an open-loop Poisson request stream through tcad_b200.serve.
def serve_stream(args, dev2d, dev3d):
    """The seeded request mix: 70% single-bias 2D MOSFET solves on meshes
    64x32..512x256, 25% warm-started 2D Id-Vg sweeps of 11..41 points, 5%
    3D tri-gate solves on meshes 64^3..128^3.  Devices are drawn from seeded
    design pools (built before the clock starts); every request is its own
    device (its own key).  Returns [(t_arrival, kind, design, points,
    report, contact)] and the pools."""
    from tcad_b200 import workloads as W
    rng = np.random.default_rng(7)
    n2, n3 = (24, 3) if args.small else (96, 6)
    pool2, pool3 = [], []
    for _ in range(n2):
        nx, ny = (int(rng.integers(64, 513)), int(rng.integers(32, 257)))
        if args.small:
            nx, ny = nx // 4, max(12, ny // 4)
        pool2.append(dict(nx=nx, ny=ny, Lg=float(rng.uniform(30e-7, 200e-7)),
                          Na=float(10 ** rng.uniform(16, 18)),
                          Nsd_peak=float(10 ** rng.uniform(19, 20))))
    for _ in range(n3):
        m = int(rng.integers(64, 129))
        dims = (m, int(rng.integers(64, 129)), int(rng.integers(64, 129)))
        if args.small:
            dims = tuple(max(12, d // 4) for d in dims)
        pool3.append(dims)
    t, out = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / args.rate))
        if t >= args.duration:
            break
        u = float(rng.uniform())
        if u < 0.70:
            d = int(rng.integers(len(pool2)))
            vg, vd = (float(x) for x in rng.uniform(0.0, 1.2, 2))
            pts = W.ramp({"gate": vg, "drain": vd}, BATCH_RAMP)
            out.append((t, "single2d", d, pts, [False] * (BATCH_RAMP - 1) + [True], "drain"))
        elif u < 0.95:
            d = int(rng.integers(len(pool2)))
            vd = float(rng.uniform(0.05, 1.0))
            npt = int(rng.integers(11, 42))
            pts = W.ramp({"drain": vd}, 2) + [{"gate": float(vg), "drain": vd}
                                              for vg in np.linspace(0.0, 1.0, npt)]
            out.append((t, "sweep2d", d, pts, [False, False] + [True] * npt, "drain"))
        else:
            d = int(rng.integers(len(pool3)))
            vg, vd = (float(x) for x in rng.uniform(0.0, 1.0, 2))
            pts = [W.trigate_bias(vd * (s + 1) / 3, vg * (s + 1) / 3) for s in range(3)]
            out.append((t, "single3d", d, pts, [False, False, True], "drain"))
    return out, pool2, pool3


def run_serve(args):
    import torch
    import tcad_b200 as tb
    from tcad_b200 import _lib
    from tcad_b200 import workloads as W
    from tcad_b200.serve import Request, Server
    lib = _lib.load()
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    stream, pool2, pool3 = serve_stream(args, tb.Device2D, tb.Device3D)
    t_build = time.perf_counter()
    setups2 = [W.mosfet2d(tb.Device2D, **q).setup for q in pool2]
    setups3 = [W.trigate3d(tb.Device3D, *d).setup for d in pool3]
    t_build = time.perf_counter() - t_build
    opts = tb.NewtonOptions(**METHODS[args.method])
    budget = args.budget_gb * 1e9
    srv = Server(budget={2: int(0.75 * budget), 3: int(0.25 * budget)}, opts=opts)
    # warm-up: one request of each kind, untimed
    srv.start()
    for kind, setups in (("2d", setups2), ("3d", setups3)):
        pts = (W.ramp({"gate": 0.5, "drain": 0.5}, 2) if kind == "2d"
               else [W.trigate_bias(0.3, 0.3)])
        srv.submit(Request(f"warm{kind}", setups[0], pts, "drain"))
    srv.wait_idle()
    for w in srv.workers.values():
        w.rounds, w.round_log, w.h2d_bytes, w.d2h_bytes = 0, [], 0, 0
    torch.cuda.synchronize()
    L0 = lib.tcad_launch_count()
    reqs = []
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        t0 = time.perf_counter()
        for q, (ta, kind, d, pts, rep, contact) in enumerate(stream):
            now = time.perf_counter() - t0
            if ta > now:
                time.sleep(ta - now)
            setup = setups2[d] if kind != "single3d" else setups3[d]
            reqs.append(srv.submit(Request(f"{kind}-{q}", setup, pts, contact, rep,
                                           arrival=t0 + ta)))
        left = max(0.0, t0 + args.duration + args.drain - time.perf_counter())
        ok = srv.wait_idle(timeout=left)
        t_end = time.perf_counter()
    srv.stop(abort=not ok)
    torch.cuda.synchronize()
    launches = lib.tcad_launch_count() - L0
    done = [r for r in reqs
            if r.finished is not None and r.error is None and r.finished <= t_end]
    pts_conv = sum(sum(r.converged) for r in done)
    pts_all = sum(r.reported_points for r in reqs)
    lat = np.array([r.latency for r in done]) * 1e3
    elapsed = t_end - t0
    by_kind = {}
    for kind in ("single2d", "sweep2d", "single3d"):
        lk = np.array([r.latency for r in done if r.key.startswith(kind)]) * 1e3
        if lk.size:
            by_kind[kind] = {"requests": int(lk.size), "p50_ms": float(np.median(lk)),
                             "p99_ms": float(np.percentile(lk, 99))}
    h2d = sum(w.h2d_bytes for w in srv.workers.values())
    d2h = sum(w.d2h_bytes for w in srv.workers.values())
    def round_stats(log):
        if not log:
            return {"rounds": 0}
        a = np.array([(t1 - t0, n, nn, it, nf, nodes, teq, kit)
                      for t0, t1, n, nn, it, nf, nodes, teq, kit in log])
        return {"rounds": len(log), "mean_instances": float(a[:, 1].mean()),
                "max_instances": int(a[:, 1].max()), "new_devices": int(a[:, 2].sum()),
                "round_s_p50": float(np.median(a[:, 0])), "round_s_max": float(a[:, 0].max()),
                "round_s_total": float(a[:, 0].sum()),
                "newton_iters_max_p50": float(np.median(a[:, 3])),
                "newton_iters_max": int(a[:, 3].max()),
                "unconverged_instances": int(a[:, 4].sum()),
                "mean_round_nodes": float(a[:, 5].mean()),
                "equilibrium_s_total": float(a[:, 6].sum()),
                "krylov_iters_max_p50": float(np.median(a[:, 7]))}
    rounds = {d: round_stats(w.round_log) for d, w in srv.workers.items()}
    value = pts_conv / elapsed

    # the plain FP64 path: the same requests in arrival order, one after another
    # through the drop-in device API, until the time cap
    popts = tb.NewtonOptions(**METHODS["plain"])
    p_pts, p_time, p_req, p_err = 0, 0.0, 0, []
    served = {r.key: r for r in reqs}
    for q, (ta, kind, d, pts, rep, contact) in enumerate(stream):
        if p_time > args.plain_seconds:
            break
        dev = (W.mosfet2d(tb.Device2D, **pool2[d]) if kind != "single3d"
               else W.trigate3d(tb.Device3D, *pool3[d]))
        torch.cuda.synchronize()
        a = time.perf_counter()
        dev.solve_equilibrium(popts)
        I = []
        for v, r_ in zip(pts, rep):
            dev.solve_bias(v, popts)
            if r_:
                I.append(dev.terminal_current(contact))
                p_pts += int(dev.last_converged)
        torch.cuda.synchronize()
        p_time += time.perf_counter() - a
        p_req += 1
        r = served[f"{kind}-{q}"]
        if r.error is None and r.currents:
            p_err.extend(abs(x - y) / max(abs(y), 1e-300)
                         for x, y, ok_ in zip(r.currents, I, r.converged) if ok_)
        dev._pack = None
    plain_rate = p_pts / p_time if p_time > 0 else None
    return {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
        "steps": len(reqs), "warmup": 2, "ms_per_step": 1e3 * elapsed / max(len(reqs), 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (FP32 inner Krylov)" if args.method == "mixed" else "f64",
        "data": "synthetic request stream (seeded Poisson arrivals, seeded device designs)",
        "config": {"workload": f"serve: Poisson {args.rate:g} req/s for {args.duration:g} s; "
                               "70% single-bias 2D MOSFET 64x32..512x256 (4-step ramp), "
                               "25% warm-started 2D Id-Vg sweeps of 11..41 points, 5% 3D "
                               "tri-gate 64^3..128^3 (3-step ramp)",
                   "method": METHOD_DESC[args.method] + "; continuous batching at bias-point "
                             "rounds over HBM arenas (2D and 3D on separate streams)",
                   "budget_gb": args.budget_gb, "parallelism": "single GPU"},
        "requests": len(reqs), "completed": len(done), "drained": bool(ok),
        "unfinished": len(reqs) - len(done),
        "converged_points": int(pts_conv), "reported_points": int(pts_all),
        "elapsed_s": elapsed, "offered_points_per_s": pts_all / args.duration,
        "p50_ms": float(np.median(lat)) if lat.size else None,
        "p99_ms": float(np.percentile(lat, 99)) if lat.size else None,
        "latency_by_kind": by_kind, "rounds": rounds,
        "plain_fp64_gpu": {"value": plain_rate, "unit": UNIT, "requests": p_req,
                           "points": p_pts, "seconds": p_time,
                           "note": "the first requests of the same stream, solved one "
                                   "after another through Device2D/Device3D"},
        "chosen_over_plain": value / plain_rate if plain_rate else None,
        "max_rel_current_err_vs_plain_fp64": float(max(p_err)) if p_err else None,
        "e2e": {"value": value, "unit": UNIT,
                "h2d_bytes_per_step": int(h2d / max(len(reqs), 1)),
                "d2h_bytes_per_step": int(d2h / max(len(reqs), 1)),
                "note": "a step is one request; arrival to completion, uploads of each "
                        "new device's arrays and bias values and the current read-back "
                        "included"},
        "gpu_launches": int(launches), "clocks": clk.summary(), "build_s": t_build,
    }


def oracle_from(dev):
    """The same device, state and BCs for the CPU oracle."""
    from oracle import OracleDevice, OracleModels
    s = dev.setup
    m = s.models
    mat = {k: getattr(s.mat, k) for k in s.mat.__dataclass_fields__ if k != "name"}
    ora = OracleDevice(s.coords, s.doping, Ntotal=s.Ntot, T=s.T,
                       models=OracleModels(m.doping_mobility, m.srh, m.auger, m.bgn),
                       material=mat)
    for name, b in dev.bcs.items():
        if b.kind == "contact":
            ora.contacts[name] = [b.nodes.copy(), b.V]
        else:
            ora.gates[name] = [b.nodes.copy(), b.kappa, b.Vfb, b.Vg, b.w.copy()]
    return ora


def cpu_costs(ora, psi, n, p, krylov_iters=10):
    """Time one full-mesh oracle Newton iteration's pieces on the host:
    assembly + Dirichlet elimination, node-block-Jacobi set-up, and the cost
    of one BiCGStab iteration (right block-Jacobi, scipy)."""
    from oracle import eliminate_csr, build_block_jacobi
    from scipy.sparse.linalg import LinearOperator, bicgstab
    t0 = time.perf_counter()
    F, J, _, _ = ora.residual_jacobian(psi, n, p)
    Jd, rhs = eliminate_csr(J, -F, ora.fixed)
    t_asm = time.perf_counter() - t0
    t0 = time.perf_counter()
    inv = build_block_jacobi(Jd, 3)
    t_bj = time.perf_counter() - t0
    nb = Jd.shape[0] // 3
    M = LinearOperator(Jd.shape, lambda v: np.einsum("nij,nj->ni", inv,
                                                     v.reshape(nb, 3)).ravel())
    t0 = time.perf_counter()
    bicgstab(Jd, rhs, rtol=1e-30, atol=0.0, maxiter=krylov_iters, M=M)
    t_it = (time.perf_counter() - t0) / krylov_iters
    return t_asm, t_bj, t_it


def cpu_baseline(dev, state, newton_iters, krylov_iters):
    """Oracle on the host cores, one full-mesh sample at `state` (psi, n, p)
    scaled to a bias point with the GPU run's own Newton and Krylov
    iteration counts."""
    try:
        os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
        ora = oracle_from(dev)
        t_asm, t_bj, t_it = cpu_costs(ora, *state)
        per_point = [nw * (t_asm + t_bj) + kr * t_it
                     for nw, kr in zip(newton_iters, krylov_iters)]
        sec = float(np.mean(per_point))
        return {"value": 1.0 / sec, "unit": UNIT, "cores": 1, "kind": "port",
                "sample": ("oracle (numpy/scipy) on the full mesh: one assembly + "
                           f"elimination ({t_asm:.2f} s), one node-block-Jacobi set-up "
                           f"({t_bj:.2f} s), 10 scipy BiCGStab iterations "
                           f"({t_it:.3f} s each); scaled to a bias point with the GPU "
                           "run's per-point Newton and BiCGStab iteration counts"),
                "sec_per_point": sec}
    except Exception as exc:      # the baseline is reported, never required
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "port",
                "sample": f"failed: {exc!r}"}


class HostDevice:
    """Device-shaped host set-up (no GPU touched): the workload builders fill
    its BCs, then the oracle takes it over."""
    dim = 3

    def __init__(self, mesh, doping, Ntotal=None, models=None, **kw):
        import tcad_b200 as tb
        from tcad_b200.pack import Setup
        coords = (mesh.x, mesh.y) if not hasattr(mesh, "z") else (mesh.x, mesh.y, mesh.z)
        self.dim = len(coords)
        self.setup = Setup(coords, doping, Ntotal=Ntotal, models=models or tb.Models(), **kw)
        self.bcs = self.setup.bcs

    def add_contact(self, name, *ijk, V=0.0):
        from tcad_b200.pack import Contact
        self.bcs[name] = Contact(self.setup.flat(*ijk), V)

    def add_gate(self, name, *ijk, tox_cm, Vfb, Vg=0.0, normal_axis="z"):
        from tcad_b200.pack import Gate
        idx = [np.atleast_1d(np.asarray(a, dtype=np.int64)) for a in ijk]
        self.bcs[name] = Gate(self.setup.flat(*ijk), self.setup.gate_kappa(tox_cm), Vfb,
                              Vg, self.setup.gate_weight(idx, normal_axis), normal_axis)


def reference_worker(workload, small, steps, warmup, wid):
    """One host process of the reference arm: its own oracle device, timed
    over warmup + steps bounded samples; returns (seconds per bias point of
    each timed step, sample description, workload description)."""
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    lanes, steps_sched, desc, contact = build_workload(workload, small, HostDevice, HostDevice)
    ora = oracle_from(lanes[0])
    lat = []
    if workload == "diode2d":
        # full solves: every step is one real warm-started bias point
        ora.solve_equilibrium()
        pts = [v[0] for v, _ in steps_sched]
        for q in range(warmup + steps):
            t0 = time.perf_counter()
            ora.solve_bias(pts[(q + wid) % len(pts)])
            ora.terminal_current(contact)
            if q >= warmup:
                lat.append(time.perf_counter() - t0)
        sample = "full oracle bias points (scipy SuperLU), warm-started sweep"
    else:
        # bounded sample: one full-mesh Newton-iteration cost per step, at the
        # bulk-guess state, scaled with the plain GPU path's iteration counts
        psi = ora.bulk_guess()
        n = ora.nie_s * np.exp(psi)
        p = ora.nie_s * np.exp(-psi)
        for q in range(warmup + steps):
            t_asm, t_bj, t_it = cpu_costs(ora, psi, n, p, krylov_iters=5)
            sec = (TRIGATE_ITERS["newton_per_point"] * (t_asm + t_bj)
                   + TRIGATE_ITERS["newton_per_point"] * TRIGATE_ITERS["krylov_per_newton"]
                   * t_it)
            if q >= warmup:
                lat.append(sec)
        sample = ("per step and process: one full-mesh oracle assembly + elimination + "
                  "node-block-Jacobi set-up + 5 scipy BiCGStab iterations, scaled to a "
                  f"bias point with {TRIGATE_ITERS['newton_per_point']} Newton x "
                  f"{TRIGATE_ITERS['krylov_per_newton']} BiCGStab iterations")
    return lat, sample, desc


def reference_processes(workload, small):
    """Host processes for the reference arm: every core, bounded by memory
    (about 3 GB per full-size 3D oracle, 0.5 GB per 2D one)."""
    cores = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 16e9
    per = 0.5e9 if (workload == "diode2d" or small) else 3.0e9
    return max(1, min(cores, int(0.7 * avail // per)))


def workload_extrapolated(workload):
    """True where the reference arm's rate is a measured per-iteration cost
    scaled to a bias point (every 3D workload: a full CPU bias point of a
    million-node device takes hours), False where each step is a full
    measured bias point (the 2D diode)."""
    return workload != "diode2d"


def run_reference(args):
    """The oracle's CPU implementation on the host cores (rank 0 only): one
    process per core, each an independent stream of bias points (the
    reference's own parallel pattern for independent points); the rate is
    the sum over processes."""
    if int(os.environ.get("RANK", "0")) != 0:
        return None
    import concurrent.futures as cf
    import multiprocessing as mp
    nproc = reference_processes(args.workload, args.small)
    with cf.ProcessPoolExecutor(nproc, mp_context=mp.get_context("spawn")) as ex:
        futs = [ex.submit(reference_worker, args.workload, args.small, args.steps,
                          args.warmup, w) for w in range(nproc)]
        outs = [f.result() for f in futs]
    lats = [np.asarray(o[0]) for o in outs]
    sample, desc = outs[0][1], outs[0][2]
    # aggregate rate of each timed step: sum over processes of 1 / seconds
    rates = np.sum([1.0 / l for l in lats], axis=0)
    value = float(np.mean(rates))
    sec = 1.0 / value
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sec, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic device",
            "config": {"workload": desc, "method": "oracle CPU port (numpy/scipy)"},
            "extrapolated": workload_extrapolated(args.workload),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": "port",
                             "sample": sample + f"; {nproc} processes x 1 thread",
                             "per_process_sec_per_point": float(np.mean(
                                 [l.mean() for l in lats]))},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_kernels(args):
    """A short, representative launch sequence for ncu: 3 coupled assemblies,
    one block-Jacobi set-up, 3 block SpMVs, one 20-iteration BiCGStab on the
    full system and one on its red-black Schur complement, on the full
    workload at its neutral-bulk state (no Newton solve)."""
    import torch
    import tcad_b200 as tb
    from tcad_b200 import _lib
    lib = _lib.load()
    lanes, _, desc, contact = build_workload(args.workload, args.small, tb.Device2D,
                                             tb.Device3D)
    dev = lanes[0]
    pk = dev.pack
    pk.set_asm_stage(args.asm_stage)
    s = dev.setup
    g = s.bulk_guess()
    pk.psi.copy_(dev._to_dev(g))
    pk.n.copy_(dev._to_dev(s.nie_s * np.exp(g)))
    pk.p.copy_(dev._to_dev(s.nie_s * np.exp(-g)))
    pk.set_bias()
    sp = _lib.stream_ptr()
    for _ in range(3):
        _lib.check(lib.tcad_sg_assemble(pk.pref, _lib.ptr(pk.psi), _lib.ptr(pk.n),
                                        _lib.ptr(pk.p), _lib.ptr(pk.F), _lib.ptr(pk.J),
                                        _lib.MODE_ELIMINATE, sp), "assemble")
    st = torch.zeros(max(1, len(pk.setups)), dtype=torch.int32, device=pk.device)
    _lib.check(lib.tcad_block_jacobi_setup(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F),
                                           _lib.ptr(st), sp), "bj")
    y = torch.empty_like(pk.du)
    for _ in range(3):
        _lib.check(lib.tcad_block_spmv(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F), _lib.ptr(y),
                                       sp), "spmv")
    it, stt, rr = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_double(0)
    _lib.check(lib.tcad_block_krylov(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F), _lib.ptr(pk.du),
                                     0, 1e-30, 20, 0, _lib.ptr(pk.work), pk.work.numel(),
                                     ctypes.byref(it), ctypes.byref(stt), ctypes.byref(rr),
                                     sp), "krylov")
    # the same 20 iterations on the red-black Schur complement
    _lib.check(lib.tcad_block_krylov(pk.pref, _lib.ptr(pk.J), _lib.ptr(pk.F), _lib.ptr(pk.du),
                                     2, 1e-30, 20, 0, _lib.ptr(pk.work), pk.work.numel(),
                                     ctypes.byref(it), ctypes.byref(stt), ctypes.byref(rr),
                                     sp), "krylov red-black")
    torch.cuda.synchronize()
    print(json.dumps({"mode": "kernels", "workload": desc, "nodes": int(dev.N),
                      "krylov_iters": it.value, "launches": int(lib.tcad_launch_count())}))


def main():
    args = parse()
    if args.no_fused and args.impl != "reference":
        from tcad_b200 import _lib
        _lib.load().tcad_set_krylov_fused(0)
    if args.kernels:
        run_kernels(args)
        return
    if args.impl == "reference":
        res = run_reference(args)
    elif args.workload == "mosfet2d_batch":
        res = run_batch(args)
    elif args.workload == "serve":
        res = run_serve(args)
    else:
        res = run_ours(args)
    if res:
        print(json.dumps(res))
        sys.stdout.flush()


if __name__ == "__main__":
    main()
