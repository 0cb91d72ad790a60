"""Benchmark: cell-steps/s of the ten Tusscher-Panfilov 2006 M-cell model
with GRL1 over 1,048,576 nodes (FP32 arithmetic, FP64 state accumulation),
with the FP64 path, the FP32-vs-FP64 V error and the end-to-end API number.

Workload (per GPU): TP06 M-cell, GRL1, internal step 0.01 ms, 1,048,576 nodes,
per-node field parameters g_Kr, g_Ks, g_CaL, g_to = default * exp(0.2 xi),
xi ~ N(0, 1) (seed 1234), initial states = IC * (1 + u), u ~ U(-0.05, 0.05),
stimulus -52 pA/pF for 1 ms at t = 10 ms (model defaults).  One bench step
is one ``forward(t, 10 ms)`` = 1000 internal steps at every node; W warm-up
steps plus K timed steps advance the model W+K times 10 ms (the default
3 + 47 covers the 500 ms of the workload).  The states (159 MB FP64) exceed
L2 (126 MB) and stay in registers inside a step, so no L2 flush is needed.

Usage::

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

MODEL = "tentusscher_panfilov_2006_M_cell"
FIELDS = ["g_Kr", "g_Ks", "g_CaL", "g_to"]
N_NODES = 1 << 20
LDT = 0.01
INTERVAL = 10.0
SEED = 1234
METRIC = "cell-steps/s tenTusscher GRL1 1M nodes: FP32 vs FP64 @V err<=1e-3; adjoint/fwd"


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=47)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="goss_b200", choices=["goss_b200", "reference"])
    ap.add_argument("--nodes", type=int, default=N_NODES)
    ap.add_argument("--skip-fp64", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--profile", choices=["single", "double", "adjoint-single", "adjoint-double", "batch"]
                    + list(_IMPLICIT_PROFILES),
                    default=None,
                    help="only run the timed forward loop in one precision, one adjoint gradient "
                         "(65,536 nodes x 2,000 steps), W+K intervals of one implicit solver on "
                         "65,536 nodes of the implicit workload, or W+K launches of a 20-forward "
                         "batch graph over the six populations at a quarter of their sizes, for ncu "
                         "captures")
    return ap.parse_args()


# --profile choice -> label of IMPLICIT_SOLVERS
_IMPLICIT_PROFILES = {"theta": "ThetaSolver", "esdirk": "ESDIRK23a", "theta-jacobian": "ThetaSolver+jacobian",
                      "ie-jacobian": "ImplicitEuler+jacobian", "esdirk-jacobian": "ESDIRK23a+jacobian"}


def profile_run(args):
    """Minimal run for profiler captures: W+K forward calls of one precision,
    one record + backward pass of the adjoint workload shortened to 20 ms, or
    W+K 0.1 ms intervals of one implicit solver on 65,536 nodes."""
    import goss_b200 as goss

    if args.profile in _IMPLICIT_PROFILES:
        label = _IMPLICIT_PROFILES[args.profile]
        _, name, ldt, _, jac, sp = next(c for c in IMPLICIT_SOLVERS if c[0] == label)
        nodes = 65_536
        md, y0, fp = implicit_inputs(nodes)
        ode = goss.ParameterizedODE(IMPLICIT_MODEL, field_parameters=IMPLICIT_FIELDS,
                                    code_params={"generate_jacobian": jac})
        solver = goss.solvers.solver_mapper[name](ode)
        solver.internal_time_step = ldt
        for k, v in sp.items():
            solver.set_parameter(k, v)
        system = goss.ODESystemSolver(nodes, solver, ode)
        system.set_states(y0)
        system.field_parameters = fp
        for k in range(args.warmup + args.steps):
            system.forward(k * IMPLICIT_DT, IMPLICIT_DT)
        print(json.dumps({"profile": args.profile, "nodes": nodes, "intervals": args.warmup + args.steps,
                          "finite": bool(np.isfinite(system.states).all())}))
        return

    if args.profile == "batch":
        rng = np.random.default_rng(SEED)
        systems = []
        for model, fps, solver_name, n in BATCH_POPS:
            n = max(3, n // 4)
            ode = goss.ParameterizedODE(model, field_parameters=fps)
            s = goss.solvers.solver_mapper[solver_name](ode)
            s.internal_time_step = LDT
            sysm = goss.ODESystemSolver(n, s, ode, precision="single")
            sysm.set_states(ode.get_ic()[None, :] * (1 + rng.uniform(-0.1, 0.1, (n, ode.num_states))))
            systems.append(sysm)
        batch = goss.BatchSolver(systems)
        batch.set_config(block=128, grid=0, schedule=0)
        batch.capture(0.0, LDT, 20)  # 20 one-step forwards, one launch
        for _ in range(args.warmup + args.steps):
            batch.replay()
        states = [s.states for s in systems]
        print(json.dumps({"profile": args.profile, "nodes": batch.total_nodes, "launches": args.warmup + args.steps,
                          "finite": bool(all(np.isfinite(y).all() for y in states))}))
        return

    if args.profile.startswith("adjoint"):
        import torch
        from goss_b200.adjoint import GRL1Trace

        precision = args.profile.split("-")[1]
        nodes = 65_536
        ode = goss.ParameterizedODE(MODEL, field_parameters=FIELDS)
        defaults = np.array([ode.get_parameter(p) for p in FIELDS])
        rng = np.random.default_rng(SEED + 1)
        fp = torch.tensor(defaults[None, :] * np.exp(0.2 * rng.standard_normal((nodes, 4))), device="cuda")
        y0 = torch.tensor(ode.get_ic()[None, :] * (1 + rng.uniform(-0.02, 0.02, (nodes, ode.num_states))),
                          device="cuda")
        tr = GRL1Trace(ode, nodes, 1.0, 100, 20, 100, precision=precision)
        v = tr.run_forward(fp, y0)
        g, _ = tr.run_backward(2 * v)
        torch.cuda.synchronize()
        print(json.dumps({"profile": args.profile, "nodes": nodes, "steps": 2000,
                          "finite": bool(torch.isfinite(g).all())}))
        return

    md, y0, fp = inputs(args.nodes)
    ode = goss.ParameterizedODE(MODEL, field_parameters=FIELDS)
    solver = goss.solvers.GRL1(ode)
    solver.internal_time_step = LDT
    system = goss.ODESystemSolver(args.nodes, solver, ode, precision=args.profile)
    system.set_states(y0)
    system.field_parameters = fp
    t = 0.0
    for _ in range(args.warmup + args.steps):
        system.forward(t, INTERVAL)
        t += INTERVAL
    print(json.dumps({"profile": args.profile, "nodes": args.nodes, "launches": args.warmup + args.steps,
                      "finite": bool(np.isfinite(system.states).all())}))


def inputs(num_nodes, rank=0):
    """Seeded states and field parameters of one rank's shard."""
    from goss_b200 import models

    md = json.loads((models.find_variant(MODEL, FIELDS) / "model.json").read_text())
    rng = np.random.default_rng(SEED + rank)
    ic = np.array(md["initial_conditions"])
    y0 = ic[None, :] * (1.0 + rng.uniform(-0.05, 0.05, (num_nodes, ic.size)))
    defaults = np.array([md["default_parameters"][i] for i in md["field_parameter_indices"]])
    fp = defaults[None, :] * np.exp(0.2 * rng.standard_normal((num_nodes, len(FIELDS))))
    return md, y0, fp


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def max_over_ranks(values, dist, device):
    """Element-wise maximum of per-rank timings over all ranks (the slowest
    rank sets the job's time); identity without a process group."""
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def side_legs(args, world):
    """Whether this run adds the one-GPU figures after the headline (GRL2,
    accuracy against the reference, batched, adjoint, implicit, coupled legs):
    at one process only, since every one of them is a per-GPU figure and under
    torchrun they would hold all N GPUs for minutes without changing."""
    return not args.skip_fp64 and world == 1


def run_gpu(args, rank, world, dist):
    import torch

    import goss_b200 as goss

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    N = args.nodes
    md, y0, fp = inputs(N, rank)
    ode = goss.ParameterizedODE(MODEL, field_parameters=FIELDS, field_states=["V"])
    iv = md["state_names"].index("V")
    stream = torch.cuda.Stream()

    def make(precision):
        solver = goss.solvers.GRL1(ode)
        solver.internal_time_step = LDT
        system = goss.ODESystemSolver(N, solver, ode, precision=precision, device=dev)
        system.set_stream(stream.cuda_stream)
        system.set_states(y0)
        system.field_parameters = fp
        return system

    def timed(system, steps, warmup, t0=0.0):
        """device time of `steps` forward calls (CUDA events on the launch stream)."""
        t = t0
        for _ in range(warmup):
            system.forward_async(t, INTERVAL)
            t += INTERVAL
        system.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            start.record(stream)
        for _ in range(steps):
            system.forward_async(t, INTERVAL)
            t += INTERVAL
        with torch.cuda.stream(stream):
            end.record(stream)
        system.synchronize()
        torch.cuda.synchronize()
        ms = start.elapsed_time(end)
        return ms, t

    steps_per_call = int(round(INTERVAL / LDT))
    out = {}
    # --- FP32 (headline) ---------------------------------------------------
    s32 = make("single")
    with ClockSampler(dev) as clocks:
        ms32, t_end = timed(s32, args.steps, args.warmup)
    # --- FP64 on the same inputs and the same number of steps --------------
    fp64_ms = None
    s64 = None
    if not args.skip_fp64:
        s64 = make("double")
        fp64_ms, _ = timed(s64, args.steps, args.warmup)
    # --- plain FP64 GPU path: one launch per internal step (states through HBM
    #     every step, as goss's PyCUDA path launches one kernel per substep),
    #     the model evaluated in its printed operation order (the arithmetic of
    #     the reference's generated model code) ---
    plain64 = None
    if not args.skip_fp64:
        sp = make("double_printed")
        t = 0.0
        for _ in range(50):
            sp.forward_async(t, LDT)
            t += LDT
        sp.synchronize()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
        for _ in range(steps_per_call):
            sp.forward_async(t, LDT)
            t += LDT
        with torch.cuda.stream(stream):
            e1.record(stream)
        sp.synchronize()
        torch.cuda.synchronize()
        plain64 = float(N) * steps_per_call / (e0.elapsed_time(e1) / 1e3)
        del sp
    out["fp64_plain_value"] = plain64
    # --- accuracy of FP32 against FP64 at the end of the run ----------------
    v32 = s32.states[:, iv]
    err = None
    if s64 is not None:
        v64 = s64.states[:, iv]
        err = float(np.max(np.abs(v32 - v64) / np.maximum(np.abs(v64), 1e-12)))
        all32, all64 = s32.states, s64.states
        state_err = np.max(np.abs(all32 - all64) / np.maximum(np.abs(all64), 1e-12), axis=0)
        out["state_max_rel_err_fp32_vs_fp64"] = {n: float(e) for n, e in zip(md["state_names"], state_err)}
        del s64
    # --- end to end through the public API with host buffers -----------------
    # (V in page-locked host memory: the step's input copied in and its result
    # copied out through the public API every step)
    e2e = make("single")
    v_host = torch.empty((N, 1), dtype=torch.float64, pin_memory=True).numpy()
    v_host[:] = y0[:, iv:iv + 1]
    t = 0.0
    for _ in range(args.warmup):
        e2e.field_states = v_host
        e2e.forward(t, INTERVAL)
        e2e.get_field_states(out=v_host)
        t += INTERVAL
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    w0 = time.perf_counter()
    for _ in range(args.steps):
        e2e.field_states = v_host          # H2D: this step's input (V), N doubles
        e2e.forward(t, INTERVAL)           # synchronous like the reference
        e2e.get_field_states(out=v_host)   # D2H: this step's result (V), N doubles
        t += INTERVAL
    e2e_s = time.perf_counter() - w0
    del e2e

    side = side_legs(args, world)
    out["grl2"] = run_grl2(dev, y0, fp) if side else None
    out["accuracy"] = run_accuracy(dev) if side and rank == 0 else None
    out["batched"] = run_batched(args, dev) if side else None
    out["adjoint"] = run_adjoint(dev) if side else None
    out["implicit"] = run_implicit(dev) if side else None
    out["coupled"] = run_coupled(dev) if side else None

    ms32, fp64_ms_max, e2e_s = max_over_ranks([ms32, fp64_ms or 0.0, e2e_s], dist, "cuda")
    cell_steps = float(N) * steps_per_call * args.steps * world
    value = cell_steps / (ms32 / 1e3)
    out.update(dict(
        value=value, ms_per_step=ms32 / args.steps, clocks=clocks.summary(),
        fp64_value=(cell_steps / (fp64_ms_max / 1e3)) if fp64_ms else None,
        fp32_over_fp64=(fp64_ms_max / ms32) if fp64_ms else None,
        v_max_rel_err_fp32_vs_fp64=err,
        e2e={"value": cell_steps / e2e_s, "unit": "cell-steps/s", "h2d_bytes_per_step": 8 * N,
             "d2h_bytes_per_step": 8 * N, "path": "ODESystemSolver.field_states / forward / get_field_states "
                                                   "(public Python API), V in page-locked host memory"},
        model_time_ms=t_end,
    ))
    return out, md


def run_grl2(dev, y0, fp, warmup=1, steps=3):
    """GRL2 (GRL2.cpp:63-86) on the headline workload (1,048,576 TP06 nodes,
    the same states and lognormal fields, forward(t, 10 ms) at 0.01 ms):
    cell-steps/s in FP32 and FP64, CUDA events on the launch stream."""
    import torch

    import goss_b200 as goss

    ode = goss.ParameterizedODE(MODEL, field_parameters=FIELDS)
    stream = torch.cuda.Stream(device=dev)
    out = {"workload": f"{MODEL} GRL2 dt=0.01ms, {y0.shape[0]} nodes, 4 lognormal field parameters, "
                       f"10 ms per step, {warmup} warm-up + {steps} timed steps", "unit": "cell-steps/s"}
    for precision in ("single", "double"):
        solver = goss.solvers.GRL2(ode)
        solver.internal_time_step = LDT
        system = goss.ODESystemSolver(y0.shape[0], solver, ode, precision=precision, device=dev)
        system.set_stream(stream.cuda_stream)
        system.set_states(y0)
        system.field_parameters = fp
        t = 0.0
        for _ in range(warmup):
            system.forward_async(t, INTERVAL)
            t += INTERVAL
        system.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            system.forward_async(t, INTERVAL)
            t += INTERVAL
        e1.record(stream)
        system.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out["fp32" if precision == "single" else "fp64"] = {
            "value": y0.shape[0] * round(INTERVAL / LDT) * steps / (ms / 1e3), "ms_per_step": ms / steps}
        del system
    out["fp32_over_fp64"] = out["fp32"]["value"] / out["fp64"]["value"]
    return out


ACCURACY_NODES, ACCURACY_MS = 4096, 500


def accuracy_subset(fp, num=ACCURACY_NODES, seed=SEED + 7):
    """Node subset of the accuracy check: for each field parameter the two
    nodes with the largest and the two with the smallest value (16 extreme
    nodes for 4 fields), then seeded random nodes up to `num`, sorted."""
    ext = []
    for k in range(fp.shape[1]):
        order = np.argsort(fp[:, k], kind="stable")
        ext += [int(i) for i in (*order[:2], *order[-2:])]
    ext = list(dict.fromkeys(ext))
    rng = np.random.default_rng(seed)
    rest = rng.choice(np.setdiff1d(np.arange(fp.shape[0]), ext), num - len(ext), replace=False)
    return np.sort(np.concatenate([np.array(ext, dtype=np.int64), rest])), ext


def _device_rows(system, n):
    """Zero-copy torch view [n, ld] of a system's FP64 device state array."""
    import torch

    ptr, ld = system.device_states()

    class _A:
        __cuda_array_interface__ = {"shape": (n, ld), "typestr": "<f8", "data": (ptr, False), "version": 3,
                                    "strides": None, "stream": None}
    return torch.as_tensor(_A(), device=torch.device("cuda", torch.cuda.current_device()))


def run_accuracy(dev, ms_total=ACCURACY_MS):
    """The 1,048,576-node lognormal workload (the headline inputs) for the full
    500 ms with GRL1 and GRL2, FP64 and FP32, against the reference's own
    compiled solvers (oracle/_ref, FP64, all host cores) on a node subset.

    Both sides make the same calls, forward(k * 1 ms, 1 ms) for k < 500
    (100 internal steps of 0.01 ms each); the GPU runs all nodes and its
    subset is gathered on the device after every call.  Reported per state:
    the worst relative error |gpu - ref| / max(|ref|, 0.01 s) over the subset
    and the 500 samples, s the state's largest magnitude in the run (the
    membrane potential passes through 0 mV in every upstroke, where an
    unfloored relative error divides rounding by ~0), and the plain relative
    error |gpu - ref| / max(|ref|, 1e-12) at the end; for FP64 also the parity
    ratio, the worst error over 1e-12 + 1e-10 max(|ref|, 0.01 s) (<= 1: within
    1e-10), over the run and at the end (1e-12 + 1e-10 |ref|).  GRL1 also runs
    in the printed operation order (GOSS_FP64_PRINTED, "fp64_printed"), to
    show what the split FP64 program changes."""
    import threading

    import torch

    import goss_b200 as goss

    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    from goss_b200 import models

    md, y0, fp = inputs(N_NODES)
    names = md["state_names"]
    n = len(names)
    idx, ext = accuracy_subset(fp)
    vdir = models.find_variant(MODEL, FIELDS)
    om = pyoracle.OracleModel(pyoracle.build_oracle(vdir, md["ident"]), md["ident"])
    plugin = pyoracle.REFDIR / vdir.name / "libplugin.so"
    kind = "reference" if pyoracle.ref_available() and plugin.exists() else "port"
    threads = cpu_threads()
    ref = {}

    def cpu_run(solver):
        if kind == "reference":
            r = pyoracle.RefSystem(plugin, md["class_name"], solver, idx.size, om.solver_params(solver, ldt=LDT))
            r.set_states(y0[idx])
            r.set_field_parameters(fp[idx])
            r.set_num_threads(threads)
            fwd, get = (lambda t: r.forward(t, 1.0)), r.get_states
        else:
            o = pyoracle.OracleSystem(om, solver, idx.size, ldt=LDT)
            o.states[:] = y0[idx]
            o.field_params[:] = fp[idx]
            fwd, get = (lambda t: o.forward(t, 1.0, threads=threads)), (lambda: o.states.copy())
        out = np.empty((ms_total, idx.size, n))
        for k in range(ms_total):
            fwd(float(k))
            out[k] = get()
        ref[solver] = out

    cpu = threading.Thread(target=lambda: [cpu_run(s) for s in ("GRL1", "GRL2")])
    w0 = time.perf_counter()
    cpu.start()
    ode = goss.ParameterizedODE(MODEL, field_parameters=FIELDS)
    gidx = torch.tensor(idx, device=torch.device("cuda", dev))
    gpu = {}
    for solver, precision in (("GRL1", "double"), ("GRL1", "single"), ("GRL1", "double_printed"),
                              ("GRL2", "double"), ("GRL2", "single")):
        s = goss.solvers.solver_mapper[solver](ode)
        s.internal_time_step = LDT
        system = goss.ODESystemSolver(N_NODES, s, ode, precision=precision, device=dev)
        system.set_states(y0)
        system.field_parameters = fp
        rows = _device_rows(system, n)
        out = np.empty((ms_total, idx.size, n))
        for k in range(ms_total):
            system.forward(float(k), 1.0)
            out[k] = rows.index_select(1, gidx).T.cpu().numpy()
        gpu[(solver, precision)] = out
        del rows, system
    cpu.join()
    wall = time.perf_counter() - w0

    def rel(a, b, floor=1e-12):
        return np.abs(a - b) / np.maximum(np.abs(b), floor)

    res = {"workload": f"{MODEL}, {N_NODES} nodes, 4 lognormal field parameters (the headline inputs), "
                       f"forward(k*1ms, 1ms) for k < {ms_total} (dt 0.01 ms)",
           "subset": f"{idx.size} nodes: the {len(ext)} nodes with the 2 largest and 2 smallest value of each "
                     f"field, then seeded random nodes",
           "reference": {"kind": kind, "cores": threads, "solver": "goss ODESystemSolver, FP64"},
           "samples": f"every 1 ms ({ms_total} samples) and the end", "wall_s": wall}
    for solver in ("GRL1", "GRL2"):
        r = ref[solver]
        floor = 0.01 * np.abs(r).max(axis=(0, 1))  # per state
        entry = {}
        for precision, key in (("double", "fp64"), ("single", "fp32"), ("double_printed", "fp64_printed")):
            if (solver, precision) not in gpu:
                continue
            g = gpu[(solver, precision)]
            e_all = rel(g, r, floor).max(axis=(0, 1))
            e_end = rel(g[-1], r[-1]).max(axis=0)
            d = {"max_rel_err": float(e_all.max()), "v_max_rel_err": float(e_all[names.index("V")]),
                 "max_rel_err_end": float(e_end.max()), "v_max_rel_err_end": float(e_end[names.index("V")]),
                 "per_state": {nm: float(e) for nm, e in zip(names, e_all)}}
            if key != "fp32":
                d["parity"] = float((np.abs(g - r) / (1e-12 + 1e-10 * np.maximum(np.abs(r), floor))).max())
                d["parity_end"] = float((np.abs(g[-1] - r[-1]) / (1e-12 + 1e-10 * np.abs(r[-1]))).max())
            entry[key] = d
        res[solver] = entry
    return res


BATCH_POPS = [  # heterogeneous workload: model, field parameters, solver, nodes
    ("fitzhughnagumo", ["a", "b"], "RK4", 3),
    ("fitzhughnagumo", ["a", "b"], "RK4", 200_000),
    ("oscilator", ["a", "b"], "RK4", 5_000),
    ("tentusscher_2004_mcell", FIELDS, "GRL1", 700_000),
    ("tentusscher_panfilov_2006_M_cell", FIELDS, "GRL1", 64_000),
    ("tentusscher_panfilov_2006_M_cell", FIELDS, "GRL1", 1_000_000),
]


def run_batched(args, dev, steps=1000, dt=0.01, precision="single"):
    """Six populations (1,969,003 nodes, 2/17/19 states, RK4 and GRL1) in one
    persistent kernel; 1000 forwards of dt = 0.01 ms captured in one CUDA
    graph, all of them in one launch (the states stay on chip between
    forwards), and the same graph with one launch per forward for comparison;
    launch configuration from the autotuner."""
    import goss_b200 as goss
    from goss_b200 import autotune

    rng = np.random.default_rng(SEED)
    systems = []
    for model, fps, solver, n in BATCH_POPS:
        ode = goss.ParameterizedODE(model, field_parameters=fps)
        s = goss.solvers.solver_mapper[solver](ode)
        s.internal_time_step = dt
        sysm = goss.ODESystemSolver(n, s, ode, precision=precision, device=dev)
        sysm.set_states(ode.get_ic()[None, :] * (1 + rng.uniform(-0.1, 0.1, (n, ode.num_states))))
        sysm.field_parameters = sysm.field_parameters * (1 + rng.uniform(-0.1, 0.1, (n, len(fps))))
        systems.append(sysm)
    batch = goss.BatchSolver(systems)
    tuned = autotune.tune_batch(batch, interval=dt, steps=20)
    batch.time(0.0, dt, 10, use_graph=False)  # warm-up
    ms = batch.time(0.0, dt, steps, use_graph=True)
    nodes = batch.total_nodes
    config = dict(batch.config)
    # the same graph with one launch per forward (states through HBM every forward)
    batch.set_config(**dict(config, forwards_per_launch=1))
    ms1 = batch.time(steps * dt, dt, steps, use_graph=True)
    batch.set_config(**config)
    return {"value": nodes * steps / (ms / 1e3), "unit": "cell-steps/s", "nodes": nodes, "forwards": steps,
            "ms": ms, "precision": precision, "graph": True, "config": config,
            "launch_per_forward": {"value": nodes * steps / (ms1 / 1e3), "ms": ms1},
            "populations": [f"{m}/{s}/{n}" for m, _, s, n in BATCH_POPS]}


def run_adjoint(dev, nodes=65_536, num_intervals=400, steps_per_interval=100, checkpoint_every=100):
    """Gradient of a V-trace misfit w.r.t. four conductance fields (adjoint).

    TP06 M-cell, GRL1 dt = 0.01 ms, 65,536 nodes, 400 ms (40,000 steps), V
    sampled every 1 ms; fields lognormal sigma 0.2 (seed A), the target trace
    from an FP64 solve with seed-B fields; loss = sum (V - V_target)^2;
    checkpoints every 100 steps, the last segments that fit in free HBM taped
    by the record pass.  Times (CUDA events on the launch stream) the FP32
    recording forward, the FP32 adjoint (with and without the tape) and, for
    the cost ratio, one plain FP32 forward solve of the same 400 ms loop
    through ODESystemSolver;
    the FP32 gradient is compared with the FP64 adjoint's (itself checked
    against the FP64 tangent-linear reference in the tests)."""
    import torch

    import goss_b200 as goss
    from goss_b200.adjoint import GRL1Trace

    ode = goss.ParameterizedODE(MODEL, field_parameters=FIELDS)
    defaults = np.array([ode.get_parameter(p) for p in FIELDS])
    rng_a, rng_b = np.random.default_rng(SEED + 1), np.random.default_rng(SEED + 2)
    fp_a = defaults[None, :] * np.exp(0.2 * rng_a.standard_normal((nodes, 4)))
    fp_b = defaults[None, :] * np.exp(0.2 * rng_b.standard_normal((nodes, 4)))
    y0 = ode.get_ic()[None, :] * (1 + rng_a.uniform(-0.02, 0.02, (nodes, ode.num_states)))
    cuda = torch.device("cuda", dev)
    fa, fb, y0t = (torch.tensor(x, device=cuda) for x in (fp_a, fp_b, y0))
    interval = steps_per_interval * LDT

    def events():
        return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def grad(tr, warm=True):
        if warm:  # one untimed forward + backward
            v = tr.run_forward(fa, y0t)
            tr.run_backward(2 * (v - target))
        torch.cuda.synchronize()
        s = torch.cuda.current_stream(cuda)
        e0, e1 = events()
        e2, e3 = events()
        e0.record(s)
        v = tr.run_forward(fa, y0t)
        e1.record(s)
        tb = 2 * (v - target)
        e2.record(s)
        g, _ = tr.run_backward(tb)
        e3.record(s)
        torch.cuda.synchronize()
        return g.cpu().numpy(), e0.elapsed_time(e1), e2.elapsed_time(e3), float(((v - target) ** 2).sum())

    def tape_bytes(tr):
        return 0 if tr._tape is None else tr._tape.numel() * tr._tape.element_size()

    # the record pass tapes as many of the last segments as the free HBM holds
    torch.cuda.empty_cache()
    tr64 = GRL1Trace(ode, nodes, interval, steps_per_interval, num_intervals, checkpoint_every, precision="double",
                     tape_bytes="auto")
    target = tr64.run_forward(fb, y0t).clone()
    g64, fwd64, bwd64, loss64 = grad(tr64, warm=False)
    tape64 = (tr64.taped_segments, tape_bytes(tr64))
    del tr64
    torch.cuda.empty_cache()
    tr32 = GRL1Trace(ode, nodes, interval, steps_per_interval, num_intervals, checkpoint_every, precision="single",
                     tape_bytes="auto")
    g32, fwd32, bwd32, loss32 = grad(tr32)
    cp_bytes = tr32._checkpoints.numel() * tr32._checkpoints.element_size()
    tape32 = (tr32.taped_segments, tape_bytes(tr32))
    del tr32
    torch.cuda.empty_cache()
    # the FP32 trajectory differentiated with FP64 step VJPs: splits the FP32
    # gradient's error into the trajectory's share and the reverse arithmetic's
    tr32m = GRL1Trace(ode, nodes, interval, steps_per_interval, num_intervals, checkpoint_every, precision="single",
                      tape_bytes="auto", reverse_precision="double")
    g32m, _, bwd32m, _ = grad(tr32m)
    del tr32m
    torch.cuda.empty_cache()
    # every segment recomputed from its checkpoint (no tape)
    tr32r = GRL1Trace(ode, nodes, interval, steps_per_interval, num_intervals, checkpoint_every, precision="single")
    g32r, fwd32r, bwd32r, _ = grad(tr32r)
    del tr32r
    torch.cuda.empty_cache()

    # one plain FP32 forward solve of the same loop (ODESystemSolver, persistent kernel per interval)
    solver = goss.solvers.GRL1(ode)
    solver.internal_time_step = LDT
    system = goss.ODESystemSolver(nodes, solver, ode, precision="single", device=dev)
    system.set_states(y0)
    system.field_parameters = fp_a
    system.forward(0.0, interval)  # warm-up
    system.set_states(y0)
    torch.cuda.synchronize()
    s = torch.cuda.current_stream(cuda)
    system.set_stream(s.cuda_stream)
    e0, e1 = events()
    e0.record(s)
    for j in range(num_intervals):
        system.forward_async(j * interval, interval)
    e1.record(s)
    system.synchronize()
    torch.cuda.synchronize()
    plain = e0.elapsed_time(e1)

    den = np.maximum(np.abs(g64).max(axis=0), 1e-300)
    col_err = np.abs(g32 - g64).max(axis=0) / den
    traj_err = np.abs(g32m - g64).max(axis=0) / den    # FP32 trajectory, FP64 VJPs vs all FP64
    rev_err = np.abs(g32 - g32m).max(axis=0) / den     # FP32 VJPs vs FP64 VJPs, same trajectory
    elem = np.abs(g32 - g64) / np.maximum(np.abs(g64), 1e-12 * den)
    return {
        "workload": f"TP06 GRL1 dt=0.01ms, {nodes} nodes, {num_intervals} ms ({num_intervals * steps_per_interval} "
                    f"steps), V every 1 ms, 4 lognormal conductance fields, checkpoints every {checkpoint_every} "
                    "steps",
        "fp32": {"forward_record_ms": fwd32, "backward_ms": bwd32, "loss": loss32,
                 "taped_segments": tape32[0], "tape_bytes": int(tape32[1])},
        "fp64": {"forward_record_ms": fwd64, "backward_ms": bwd64, "loss": loss64,
                 "taped_segments": tape64[0], "tape_bytes": int(tape64[1]),
                 "gradient_over_record": (fwd64 + bwd64) / fwd64},
        "segments": -(-num_intervals * steps_per_interval // checkpoint_every),
        "plain_forward_fp32_ms": plain,
        "backward_over_plain_forward": bwd32 / plain,
        "gradient_over_plain_forward": (fwd32 + bwd32) / plain,
        "fp32_recompute_all": {"forward_record_ms": fwd32r, "backward_ms": bwd32r,
                               "gradient_over_plain_forward": (fwd32r + bwd32r) / plain,
                               "max_rel_diff_vs_taped": float(np.abs(g32 - g32r).max() / np.abs(g32r).max())},
        "checkpoint_bytes_fp32": int(cp_bytes),
        "grad_rel_err_fp32_vs_fp64": {"per_field_scaled_max": {f: float(e) for f, e in zip(FIELDS, col_err)},
                                      "elementwise_median": float(np.median(elem)),
                                      "elementwise_p99": float(np.quantile(elem, 0.99)),
                                      "split": {
                                          "trajectory_part": {f: float(e) for f, e in zip(FIELDS, traj_err)},
                                          "reverse_arithmetic_part": {f: float(e) for f, e in zip(FIELDS, rev_err)},
                                          "how": "trajectory part: FP32 record + FP64 step VJPs vs the FP64 "
                                                 "adjoint; reverse part: FP32 adjoint vs FP32 record + FP64 "
                                                 "step VJPs (field-scaled max)",
                                          "fp64_vjp_backward_ms": bwd32m}},
    }


def run_coupled(dev, steps=200, pde_dt=0.1):
    """Operator splitting on the headline population: 1,048,576 TP06 nodes,
    FP32 GRL1 at 0.01 ms, V exchanged with a PDE vector every 0.1 ms (10
    internal steps per exchange), 200 exchanges.  Device: FieldStateCoupling
    (PDE vector a CUDA tensor, zero-copy exchange on the launch stream);
    host: the reference's way, field states copied to and from a host vector
    every exchange.  No PDE work in either, so the difference is the exchange."""
    import torch

    import goss_b200 as goss
    from goss_b200.coupling import FieldStateCoupling

    md, y0, fp = inputs(N_NODES)
    ode = goss.ParameterizedODE(MODEL, field_parameters=FIELDS, field_states=["V"])
    iv = md["state_names"].index("V")

    def make():
        solver = goss.solvers.GRL1(ode)
        solver.internal_time_step = LDT
        system = goss.ODESystemSolver(N_NODES, solver, ode, precision="single", device=dev)
        system.set_states(y0)
        system.field_parameters = fp
        return system

    out = {}
    system = make()
    cpl = FieldStateCoupling({"tissue": system}, {"tissue": np.arange(N_NODES)}, N_NODES)
    v = torch.tensor(y0[:, iv], device=torch.device("cuda", dev))
    for k in range(5):
        cpl.step((k * pde_dt, (k + 1) * pde_dt), v)
    cpl.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(cpl.stream)
    for k in range(5, 5 + steps):
        cpl.step((k * pde_dt, (k + 1) * pde_dt), v)
    e1.record(cpl.stream)
    cpl.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    cell_steps = float(N_NODES) * steps * round(pde_dt / LDT)
    out["device"] = {"value": cell_steps / (ms / 1e3), "ms_per_exchange": ms / steps}
    del cpl, system
    system = make()
    vh = torch.empty((N_NODES, 1), dtype=torch.float64, pin_memory=True).numpy()
    vh[:] = y0[:, iv:iv + 1]
    for k in range(5):
        system.field_states = vh
        system.forward(k * pde_dt, pde_dt)
        system.get_field_states(out=vh)
    w0 = time.perf_counter()
    for k in range(5, 5 + steps):
        system.field_states = vh
        system.forward(k * pde_dt, pde_dt)
        system.get_field_states(out=vh)
    s = time.perf_counter() - w0
    out["host_copies"] = {"value": cell_steps / s, "ms_per_exchange": 1e3 * s / steps}
    out["workload"] = (f"{MODEL} FP32 GRL1 dt=0.01ms, {N_NODES} nodes, V exchanged every {pde_dt} ms, "
                       f"{steps} exchanges")
    out["unit"] = "cell-steps/s"
    return out


IMPLICIT_MODEL, IMPLICIT_FIELDS, IMPLICIT_NODES, IMPLICIT_DT = "tentusscher_2004_mcell", ["g_Kr", "g_CaL"], 262_144, 0.1
# label, solver, internal step, timed intervals, analytic Jacobian (code_params generate_jacobian)
# label, solver, internal step, timed intervals, analytic Jacobian, solver parameters.
# ESDIRK23a runs with min_dt = 1e-4 ms: at the default 1e-3 ms it never accepts a
# TT04 step (its first attempt at min_dt fails the error test and the step size
# cannot shrink further -- the reference behaves the same), so the default
# configuration times rejected attempts only ("min_dt 1e-3" rows).
ESDIRK_MIN_DT = 1e-4
IMPLICIT_SOLVERS = [("ThetaSolver", "ThetaSolver", 0.1, 10, False, {}),
                    ("ESDIRK23a", "ESDIRK23a", -1.0, 10, False, {"min_dt": ESDIRK_MIN_DT}),
                    ("ThetaSolver+jacobian", "ThetaSolver", 0.1, 20, True, {}),
                    ("ImplicitEuler+jacobian", "ImplicitEuler", 0.1, 20, True, {}),
                    ("ESDIRK23a+jacobian", "ESDIRK23a", -1.0, 10, True, {"min_dt": ESDIRK_MIN_DT}),
                    ("ESDIRK23a min_dt 1e-3", "ESDIRK23a", -1.0, 2, False, {}),
                    ("ESDIRK23a+jacobian min_dt 1e-3", "ESDIRK23a", -1.0, 2, True, {})]


def implicit_inputs(nodes):
    """TT04 M-cell states IC*(1+u), field parameters default*(1+u), u ~ U(+-5%) (seed 1234)."""
    from goss_b200 import models

    md = json.loads((models.find_variant(IMPLICIT_MODEL, IMPLICIT_FIELDS) / "model.json").read_text())
    rng = np.random.default_rng(SEED)
    ic = np.array(md["initial_conditions"])
    y0 = ic[None, :] * (1.0 + rng.uniform(-0.05, 0.05, (nodes, ic.size)))
    defaults = np.array([md["default_parameters"][i] for i in md["field_parameter_indices"]])
    fp = defaults[None, :] * (1.0 + rng.uniform(-0.05, 0.05, (nodes, len(IMPLICIT_FIELDS))))
    return md, y0, fp


def run_implicit(dev):
    """ThetaSolver (theta 0.5, one 0.1 ms step per interval) and ESDIRK23a
    (adaptive) on TT04 M-cell, 262,144 nodes, FP64 Newton and LU, forward
    (t, 0.1 ms) per step; one untimed interval first.  Unit: node-intervals/s.
    ESDIRK23a is timed with min_dt = 1e-4 ms, where it accepts steps; with the
    reference's default min_dt (0.001 ms) it rejects every TT04 step and the
    states do not advance -- the reference's own behaviour, reproduced -- so
    those rows time 100 rejected attempts per interval."""
    import torch

    import goss_b200 as goss

    md, y0, fp = implicit_inputs(IMPLICIT_NODES)
    odes = {jac: goss.ParameterizedODE(IMPLICIT_MODEL, field_parameters=IMPLICIT_FIELDS,
                                       code_params={"generate_jacobian": jac}) for jac in (False, True)}
    stream = torch.cuda.current_stream(dev)
    out = {}
    for label, name, ldt, intervals, jac, sp in IMPLICIT_SOLVERS:
        ode = odes[jac]
        solver = goss.solvers.solver_mapper[name](ode)
        solver.internal_time_step = ldt
        for k, v in sp.items():
            solver.set_parameter(k, v)
        system = goss.ODESystemSolver(IMPLICIT_NODES, solver, ode, device=dev)
        system.set_stream(stream.cuda_stream)
        system.set_states(y0)
        system.field_parameters = fp
        system.forward(0.0, IMPLICIT_DT)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t = IMPLICIT_DT
        e0.record(stream)
        for _ in range(intervals):
            system.forward_async(t, IMPLICIT_DT)
            t += IMPLICIT_DT
        e1.record(stream)
        system.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        jac, rej, acc = system.counters()
        out[label] = {"value": IMPLICIT_NODES * intervals / (ms / 1e3), "unit": "node-intervals/s",
                     "ms_per_interval": ms / intervals, "intervals": intervals, "internal_time_step": ldt,
                     "solver_parameters": sp,
                     "jacobians_per_node_interval": float(np.mean(jac)) / (intervals + 1),
                     "rejected_per_node_interval": float(np.mean(rej)) / (intervals + 1),
                     "accepted_per_node_interval": float(np.mean(acc)) / (intervals + 1)}
        del system
    return {"workload": f"{IMPLICIT_MODEL} [g_Kr, g_CaL] U(+-5%), {IMPLICIT_NODES} nodes, forward(t, 0.1 ms), FP64",
            **out}


def implicit_reference_sample(target_s=3.0):
    """The reference's ThetaSolver / ESDIRK23a (one solver per node, OpenMP)
    on a node subset of the implicit workload: node-intervals/s."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    from goss_b200 import models

    threads = cpu_threads()
    out = {}
    for label, name, ldt, _, jac, sp in IMPLICIT_SOLVERS:
        vdir = models.find_variant(IMPLICIT_MODEL, IMPLICIT_FIELDS, jacobian=jac)
        md = json.loads((vdir / "model.json").read_text())
        om = pyoracle.OracleModel(pyoracle.build_oracle(vdir, md["ident"]), md["ident"])
        plugin = pyoracle.REFDIR / vdir.name / "libplugin.so"
        kind = "reference" if pyoracle.ref_available() and plugin.exists() else "port"
        nodes = threads * 4
        for attempt in range(2):
            _, y0, fp = implicit_inputs(nodes)
            if kind == "reference":
                r = pyoracle.RefSystem(plugin, md["class_name"], name, nodes, om.solver_params(name, ldt=ldt, **sp))
                r.set_states(y0)
                r.set_field_parameters(fp)
                r.set_num_threads(threads)
                fwd = lambda t: r.forward(t, IMPLICIT_DT)
            else:
                o = pyoracle.OracleSystem(om, name, nodes, ldt=ldt, **sp)
                o.states[:] = y0
                o.field_params[:] = fp
                fwd = lambda t: o.forward(t, IMPLICIT_DT, threads=threads)
            fwd(0.0)
            t0 = time.perf_counter()
            fwd(IMPLICIT_DT)
            dt = time.perf_counter() - t0
            if attempt == 0:
                nodes = int(min(max(nodes * target_s / max(dt, 1e-6), nodes), IMPLICIT_NODES))
                nodes = max(threads, nodes // threads * threads)
        out[label] = {"value": nodes / dt, "unit": "node-intervals/s", "kind": kind, "cores": threads,
                     "sample": f"{nodes} nodes x one 0.1 ms interval after one untimed interval, {dt:.1f} s"}
    return out


def measured_peaks(dev):
    """XU-pipe, FP32-FMA and FP64-FMA peaks of this GPU (goss_measure_peaks,
    goss_measure_fp64_peak), or None."""
    import ctypes as C

    from goss_b200 import _capi

    xu, fp, f64 = C.c_double(0.0), C.c_double(0.0), C.c_double(0.0)
    try:
        if _capi.lib().goss_measure_peaks(int(dev), C.byref(xu), C.byref(fp)) != 0:
            return None
        if _capi.lib().goss_measure_fp64_peak(int(dev), C.byref(f64)) != 0:
            f64.value = 0.0
    except Exception:
        return None
    return {"xu_ops_per_s": xu.value, "fp32_ops_per_s": fp.value, "fp64_fma_per_s": f64.value}


# FP64-pipe instructions per TP06 GRL1 cell-step of explicit_kernel<TP06, double,
# GRL1> (split program): the thread-level dadd + dmul + dfma counts of one ncu
# capture of `bench.py --profile double --steps 1 --warmup 1 --nodes 262144`
# divided by the cell-steps of the launch (262,144 x 1000)
FP64_PIPE_OPS_PER_CELL_STEP = 1962.0  # dadd 262 + dmul 371 + dfma 1329 (B200, ncu)


def roofline_fp64(value_fp64, peaks):
    """FP64 GRL1 against the measured FP64 FMA peak: FP64-pipe instructions
    per cell-step (ncu) x cell-steps/s over FP64 FMAs/s of independent chains
    (one instruction each, like a dadd or dmul)."""
    peak = (peaks or {}).get("fp64_fma_per_s") or None
    ops = FP64_PIPE_OPS_PER_CELL_STEP
    out = {"bound": "fp64 pipe", "unit": "Gop/s (FP64 pipe)", "peak": peak / 1e9 if peak else None,
           "ops_per_cell_step": ops,
           "peak_source": "measured on this GPU by goss_measure_fp64_peak (independent fma.rn.f64 chains, "
                          "2048 threads per SM)",
           "ops_source": "ncu smsp__sass_thread_inst_executed_op_{dadd,dmul,dfma}_pred_on.sum of one "
                         "explicit_kernel<TP06, double, GRL1> launch / its cell-steps"}
    if ops and peak and value_fp64:
        out["achieved"] = ops * value_fp64 / 1e9
        out["frac"] = ops * value_fp64 / peak
    return out


def roofline(md, value_fp32, ms_per_step, n_nodes, peaks=None):
    """Operation census of one GRL1 step (generator) against the CUDA-core peaks.

    The census is the generator's count of one linearised evaluation as the
    kernel runs it (``op_census.linearized_split``: parameter-only terms folded,
    every distinct exp/log/sqrt/reciprocal once) plus the GRL update (GRL1.h:
    72-84), whose algorithm takes one exponential exp(a_i h) per state.  MUFU
    (SFU) ops: exp, log, sqrt, pow (2), one reciprocal per division, and the n
    exponentials of the update (the kernel evaluates them through phi1: a
    polynomial on the FP32 pipe for |a h| < 1/4, ex2 and a reciprocal above;
    ncu counts 131 XU instructions per TP06 step in all, against 129 here).
    FP32-pipe ops: adds, muls, the multiply of every division and exponential,
    and ~10 ops of the phi1 update per state."""
    census = md["op_census"]
    lin = census.get("linearized_split", census["linearized"])
    n = len(md["state_names"])
    sfu = lin["exp"] + lin["log"] + lin["sqrt"] + 2 * lin["pow"] + lin["div"] + n
    fp = lin["add"] + lin["mul"] + lin["div"] + lin["exp"] + 10 * n
    sm_clock = 1.965e9
    nominal_sfu = 148 * 16 * sm_clock       # 16 MUFU results / clk / SM
    nominal_fma = 148 * 128 * sm_clock      # 128 FP32 lanes / clk / SM (ops, FMA = 1 op)
    measured = bool(peaks and peaks["xu_ops_per_s"] > 0 and peaks["fp32_ops_per_s"] > 0)
    sfu_peak = peaks["xu_ops_per_s"] if measured else nominal_sfu
    fma_peak = peaks["fp32_ops_per_s"] if measured else nominal_fma
    sfu_rate = sfu * value_fp32
    fp_rate = fp * value_fp32
    hbm_bytes = n_nodes * (2 * n * 8 + 4 * 8)  # states in+out, field params in, per launch
    # dram__bytes_read.sum + dram__bytes_write.sum of one launch of this kernel
    # (explicit_kernel<TP06, float, GRL1>, 1,048,576 nodes x 1000 steps) in an
    # ncu --set full capture of `bench.py --profile single --steps 1 --warmup 1`
    # on a B200: 196 MB read, 103 MB written (below the algorithmic bytes:
    # part of the states stay in L2 from the previous launch)
    ncu_dram_bytes = (196e6 + 103e6) * n_nodes / 1_048_576
    return dict(
        bound="sfu",
        achieved=sfu_rate / 1e9, peak=sfu_peak / 1e9, unit="Gop/s (MUFU)", frac=sfu_rate / sfu_peak,
        traffic=ncu_dram_bytes,
        traffic_source="ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, one capture of "
                       "bench.py --profile single (scaled by nodes when --nodes differs)",
        per_cell_step={"sfu_ops": sfu, "fp32_ops": fp},
        fp32_pipe={"achieved": fp_rate / 1e12, "peak": fma_peak / 1e12, "unit": "Top/s",
                   "frac": fp_rate / fma_peak},
        hbm={"achieved_gbs": hbm_bytes / (ms_per_step / 1e3) / 1e9, "algorithmic_bytes_per_launch": hbm_bytes},
        peak_source=("measured on this GPU after the timed region by goss_measure_peaks (independent ex2/lg2 "
                     "chains for the XU pipe, FP32 FMA chains, 2048 threads per SM)") if measured else
                    ("nominal B200: 148 SMs x (16 MUFU | 128 FP32) per clk x 1.965 GHz (no CUDA-core peak "
                     "in MEASURED_PEAKS.json)"),
        nominal_peaks={"xu_gops": nominal_sfu / 1e9, "fp32_tops": nominal_fma / 1e12},
    )


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own solvers (oracle/_ref) on a node sample
# ---------------------------------------------------------------------------
def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_sample(target_s=5.0, warmup=3):
    """Time the reference ODESystemSolver (GRL1, OpenMP over nodes) on a
    seeded node subset for one 10 ms interval, the one the GPU arm's first
    timed step covers ([10 W, 10 W + 10) ms after W untimed intervals, so both
    arms time the same phase of the model); returns cell-steps/s."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle
    from goss_b200 import models

    vdir = models.find_variant(MODEL, FIELDS)
    md = json.loads((vdir / "model.json").read_text())
    threads = cpu_threads()
    kind = "reference"
    if pyoracle.ref_available() and (pyoracle.REFDIR / vdir.name / "libplugin.so").exists():
        def make(nodes):
            om = pyoracle.OracleModel(pyoracle.build_oracle(vdir, md["ident"]), md["ident"])
            r = pyoracle.RefSystem(pyoracle.REFDIR / vdir.name / "libplugin.so", md["class_name"], "GRL1", nodes,
                                   om.solver_params("GRL1", ldt=LDT))
            _, y0, fp = inputs(nodes)
            r.set_states(y0)
            r.set_field_parameters(fp)
            r.set_num_threads(threads)
            return r, (lambda t: r.forward(t, INTERVAL))
    else:
        kind = "port"

        def make(nodes):
            om = pyoracle.OracleModel(pyoracle.build_oracle(vdir, md["ident"]), md["ident"])
            o = pyoracle.OracleSystem(om, "GRL1", nodes, ldt=LDT)
            _, y0, fp = inputs(nodes)
            o.states[:] = y0
            o.field_params[:] = fp
            return o, (lambda t: o.forward(t, INTERVAL, threads=threads))
    steps = int(round(INTERVAL / LDT))
    # calibrate on a small sample, then size the sample to ~target_s
    nodes = max(threads * 8, 256)
    obj, fwd = make(nodes)
    t0 = time.perf_counter()
    fwd(0.0)
    dt = time.perf_counter() - t0
    rate = nodes * steps / dt
    nodes = int(min(max(rate * target_s / steps, nodes), N_NODES))
    nodes = max(threads, nodes // threads * threads)
    obj, fwd = make(nodes)
    if warmup:  # untimed: [0, 10 W) ms in one call
        if kind == "reference":
            obj.forward(0.0, warmup * INTERVAL)
        else:
            obj.forward(0.0, warmup * INTERVAL, threads=threads)
    t_start = warmup * INTERVAL
    t0 = time.perf_counter()
    fwd(t_start)
    dt = time.perf_counter() - t0
    return dict(value=nodes * steps / dt, unit="cell-steps/s", cores=threads, kind=kind,
                sample=f"{nodes} seeded nodes of the workload x the 10 ms interval [{t_start:g}, "
                       f"{t_start + INTERVAL:g}) ms (1000 GRL1 steps) after {warmup} untimed intervals, "
                       f"FP64, {threads} OpenMP threads, {dt:.1f} s")


def main():
    args = _args()
    if args.profile:
        profile_run(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    config = {"workload": "tentusscher_panfilov_2006_M_cell GRL1 dt=0.01ms, 1,048,576 nodes per GPU, "
                          "4 lognormal field parameters, 10 ms per step",
              "model": MODEL, "solver": "GRL1", "nodes_per_gpu": args.nodes, "internal_dt_ms": LDT,
              "interval_ms": INTERVAL, "global_batch": args.nodes * world,
              "parallelism": f"node shards x{world}", "l2": "inputs larger than L2 (159 MB FP64 states)"}

    if args.impl == "reference":
        if rank != 0:
            return
        res = reference_sample(warmup=args.warmup)
        steps_done = 0
        line = {"metric": METRIC, "value": res["value"], "unit": "cell-steps/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                "config": config, "impl": "reference",
                "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": res["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        del steps_done
        print(json.dumps(line))
        return

    dist = None
    if world > 1:
        import torch.distributed as _dist
        from datetime import timedelta

        _dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        dist = _dist
    res, md = run_gpu(args, rank, world, dist)
    cpu = None
    if rank == 0 and world == 1:
        try:
            cpu = reference_sample(warmup=args.warmup)
        except Exception as exc:  # the baseline is reported, never the target
            cpu = {"value": None, "unit": "cell-steps/s", "cores": cpu_threads(), "kind": "reference",
                   "sample": f"failed: {exc}"}
        if not args.skip_fp64:
            try:
                cpu["implicit"] = implicit_reference_sample()
            except Exception as exc:
                cpu["implicit"] = {"failed": str(exc)}
    if rank == 0:
        peaks = measured_peaks(int(os.environ.get("LOCAL_RANK", 0)))
        rl = roofline(md, res["value"] / world, res["ms_per_step"], args.nodes, peaks)
        acc = res.get("accuracy")
        if acc:
            # the worst cases of the accuracy check, in the config block that
            # summaries of the line keep
            config["accuracy_vs_cpu_reference"] = {
                "fp64_max_rel_err": max(acc[s]["fp64"]["max_rel_err"] for s in ("GRL1", "GRL2")),
                "fp64_parity_1e-10": max(acc[s]["fp64"]["parity"] for s in ("GRL1", "GRL2")),
                "fp32_v_max_rel_err": max(acc[s]["fp32"]["v_max_rel_err"] for s in ("GRL1", "GRL2")),
                "fp32_any_state_max_rel_err": max(acc[s]["fp32"]["max_rel_err"] for s in ("GRL1", "GRL2")),
                "how": "GRL1 and GRL2, 1,048,576 nodes x 500 ms on the GPU; 4096-node subset incl. the 16 "
                       "extreme-field nodes vs the reference's compiled solvers, every 1 ms; relative to "
                       "max(|ref|, 1% of the state's largest magnitude)"}
        line = {"metric": METRIC, "value": res["value"], "unit": "cell-steps/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 states)",
                "data": "synthetic (seeded)", "config": config, "roofline": rl, "cpu_baseline": cpu,
                "e2e": res["e2e"], "gpu_launches": args.steps, "clocks": res["clocks"],
                "fp64": {"value": res["fp64_value"], "fp32_over_fp64": res["fp32_over_fp64"],
                         "plain_value": res["fp64_plain_value"],
                         "fp32_over_plain_fp64": (res["value"] / world / res["fp64_plain_value"])
                         if res["fp64_plain_value"] else None,
                         "plain_path": "one launch per 0.01 ms step, the model in its printed operation "
                                       "order (GOSS_FP64_PRINTED)",
                         "v_max_rel_err_fp32_vs_fp64": res["v_max_rel_err_fp32_vs_fp64"],
                         "roofline": roofline_fp64(res["fp64_value"] / world if res["fp64_value"] else None,
                                                   peaks)},
                "grl2": res.get("grl2"),
                "state_max_rel_err_fp32_vs_fp64": res.get("state_max_rel_err_fp32_vs_fp64"),
                "batched_heterogeneous": res.get("batched"), "adjoint": res.get("adjoint"),
                "implicit": res.get("implicit"), "coupled": res.get("coupled"),
                # last, so that the end of the line shows it in full
                "accuracy_vs_cpu_reference": res.get("accuracy")}
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
