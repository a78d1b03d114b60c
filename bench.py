#!/usr/bin/env python
"""Benchmark: RK cell-updates/s (FP64) of the COREFL per-stage RHS + update.

Workload: 3-D viscous single-species wave on a curvilinear single block of
257^3 nodes (256^3 unique points, node-periodic in all directions),
x = xi + 0.05 sin(2 pi eta) sin(2 pi zeta), rho = 1 + 0.01 sin(2 pi x), u = 1,
p = 1/gamma, Sutherland viscosity at Re = 1000, WENO7 characteristic
(inviscid_scheme 72) + second-order viscous flux, SSP-RK3 with the CFL step
(CFL 0.5) computed on the device every step.  One "step" is one full
three-stage RK3 step of the block; the metric counts nodes x steps / s.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's algorithm on the host cores (the CPU
oracle, all threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "corefl-cpc_b200"))

import numpy as np  # noqa: E402

import cases  # noqa: E402

METRIC = "RK cell-updates/s (FP64)"
UNIT = "cell-updates/s"
N_NODES = 257

# FP64 operations of one WENO7 characteristic face flux (air) with its share
# of the staging and flux difference, counted by the hardware: 2 x DFMA + DADD
# + DMUL per face from ncu's instruction counters on a 161^3 block
# (profiles/weno_air_flux_diff_161_fp64_counts.md; the same in all three
# sweeps).  It includes the FMA/multiply steps into which divisions and square
# roots expand.  The hand count of the restated arithmetic (each +, -, *, /,
# sqrt = 1; fma = 2) is 2980: face set-up 93; per characteristic field the left
# eigenvector row 14, projection of 8 points 186, two WENO7-Z sides 361, times
# 5 fields; back-projection 44; staging share 30, difference share 10.
FLOPS_PER_FACE_WENO7_CH = 3214.9
FLOPS_PER_FACE_WENO7_CH_HAND = 2980.0


# The reference's own CUDA kernels (its sources built unmodified for sm_100a,
# oracle/ref/) timed on a B200 on the same 257^3 workload by
# oracle/ref/time_ref_gpu.py: a recorded figure, stated beside the live one
# (profiles/reference_build_rk3_257_and_reactors.md).
REFERENCE_GPU_257 = {"ms_per_step": 69.84, "cell_updates_per_s": 2.43e8, "kind": "recorded",
                     "what": "reference sources built unmodified for sm_100a, RK3 loop body with its own CFL "
                             "step, median of 10 timed steps after 3 on one B200",
                     "source": "profiles/reference_build_rk3_257_and_reactors.md"}

WENO_PROFILE = os.path.join(ROOT, "profiles", "weno_air_flux_diff_161.md")
WENO_PROFILE_NODES = 161 ** 3


def weno_traffic_per_launch(nodes):
    """DRAM bytes per launch of the WENO sweep kernel: the mean of the
    'DRAM read + write per launch' row (MB, one value per sweep) of the ncu
    summary captured on a 161^3 block, scaled to `nodes` interior nodes (the
    kernel reads each input about once, so its traffic grows with the
    nodes).  Returns (bytes or None, description)."""
    try:
        with open(WENO_PROFILE) as f:
            row = next(line for line in f if line.startswith("| DRAM read + write per launch"))
        mb = [float(c.strip().split()[0]) for c in row.strip().strip("|").split("|")[1:]]
        per_launch = sum(mb) / len(mb) * 1e6 * nodes / WENO_PROFILE_NODES
        return per_launch, (f"ncu dram__bytes_read+write on 161^3 ({sum(mb) / len(mb):.0f} MB per sweep, "
                            f"profiles/weno_air_flux_diff_161.md) scaled by nodes")
    except (OSError, StopIteration, ValueError, IndexError):
        return None, "no ncu summary"


def max_over_ranks(x: float, dist, device) -> float:
    """The largest of each rank's x (one all-reduce); x itself without a process group."""
    if not dist:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def _upload(ctx, zone, case):
    """Copy metric, jac and the initial bv of the case into the context's zone."""
    for name, arr in (("metric", case.metric), ("jac", case.jac), ("bv", case.bv)):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        ctx.h2d(getattr(zone, name), a.ctypes.data, a.nbytes)
    ctx.sync()


def _cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline_sample(scheme: int, reconstruction: int, steps: int = 3, warm: int = 1, n: int = N_NODES,
                        case=None):
    """The oracle (the reference's algorithm restated in C, OpenMP on all host
    threads, built with -march=native for this host) on the workload itself:
    the n^3 wave (the benchmark block by default), `warm` untimed RK3 steps,
    then `steps` steps each timed on its own; the value is the median
    per-step rate (with the spread)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle  # test/baseline infrastructure only

    native = pyoracle.use_native_build() if pyoracle._lib is None else pyoracle.LIB_PATH.endswith("_native/liboracle.so")
    if case is None:
        case = cases.sine_wave(n=n, scheme=scheme, viscous=True, cfl=0.5, reconstruction=reconstruction)
    z = pyoracle.OracleZone(case)
    z.initialize()
    for _ in range(warm):
        z.step()
    per = []
    for _ in range(steps):
        t0 = time.perf_counter()
        z.step()
        per.append(time.perf_counter() - t0)
    rates = sorted(case.N / t for t in per)
    med = float(np.median(rates))
    del z
    return {"value": med, "unit": UNIT, "cores": int(pyoracle.lib().orc_num_threads()), "kind": "port",
            "sample": f"{case.mx}x{case.my}x{case.mz}-node block of the workload, WENO{scheme // 10 if scheme > 10 else ''}"
                      f"{'-ch' if scheme > 10 else ''} + viscous, median of {steps} RK3 steps after {warm} untimed "
                      f"(per-step rates {rates[0]:.3e}..{rates[-1]:.3e}); {'-march=native' if native else 'portable x86-64-v3'} "
                      f"build on {_cpu_model()}",
            "steps": steps, "seconds": float(sum(per)), "spread": [rates[0], rates[-1]], "cpu": _cpu_model()}


def run_reference(args, rank, world):
    if rank != 0:
        return
    # each timed step is one RK3 step of the full workload on the host
    res = cpu_baseline_sample(args.scheme, args.reconstruction, steps=max(args.steps, 1),
                              warm=min(max(args.warmup, 0), 1), n=args.n)
    line = {
        "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * res["seconds"] / max(res["steps"], 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": "3-D viscous sine wave, curvilinear periodic block, WENO7-ch + 2nd-order viscous, "
                               "SSP-RK3 CFL 0.5", "nodes": f"{args.n}^3"},
        "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def reacting_bench(args, local, world, dist):
    """Batched constant-volume H2/air chemistry: 2^20 independent reactors
    (Li-2004, 9 species / 19 reactions; T ~ U[1000,1600] K, p log-uniform in
    [1,10] atm, phi ~ U[0.5,2]) advanced by the point-implicit Wu reaction
    step, dt = 1e-7 s per step, with the two schedules: one thread per node
    and the persistent work-queue kernel.  Metric: reacting cell-steps/s."""
    import torch
    import corefl_b200 as cfk
    import mechanism

    mech = mechanism.load("li2004")
    case = cases.reactor_batch(mech, args.reacting_cells, seed=2026)
    out = {"workload": f"{case.N} constant-volume H2/air reactors, Li-2004 9s/19r, point-implicit Wu substeps, "
                       "dt 1e-7 s", "cells": case.N, "dtype": "f64"}
    nsub = torch.zeros(case.N, dtype=torch.int32, device=f"cuda:{local}")
    for name, sched in (("plain", 0), ("work_queue", 1)):
        param = dict(case.param)
        param["device"] = local
        ctx = cfk.Context(param, case.faces)
        zone = ctx.alloc_zone(case.mx, case.my, case.mz)
        ctx.set_mechanism(mech)
        for fld, arr in (("bv", case.bv), ("sv", case.sv), ("jac", case.jac), ("metric", case.metric)):
            a = np.ascontiguousarray(arr)
            ctx.h2d(getattr(zone, fld), a.ctypes.data, a.nbytes)
        ctx.cv_from_bv()
        for _ in range(args.warmup):
            ctx.wu_reaction_step(1e-7, schedule=sched)
        ctx.sync()
        if dist:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        k = max(args.steps // 2, 3)
        for _ in range(k):
            ctx.wu_reaction_step(1e-7, schedule=sched, nsub_ptr=nsub.data_ptr())
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        ms = max_over_ranks(ms, dist, f"cuda:{local}")
        n = nsub.cpu().numpy()
        out[name] = {"cells_per_s": case.N * k * world / (ms * 1e-3), "ms_per_step": ms / k, "steps": k,
                     "substeps_mean": float(n.mean()), "substeps_max": int(n.max())}
        ctx.close()
    out["speedup_work_queue"] = out["work_queue"]["cells_per_s"] / out["plain"]["cells_per_s"]
    return out


def _reactor_ctx(mech, case, local, seed):
    """A chemistry context holding `case` (constant-volume reactors) with the
    surrogate initialised."""
    import corefl_b200 as cfk
    param = dict(case.param)
    param["device"] = local
    ctx = cfk.Context(param, case.faces)
    zone = ctx.alloc_zone(case.mx, case.my, case.mz)
    ctx.set_mechanism(mech)
    for fld, arr in (("bv", case.bv), ("sv", case.sv), ("jac", case.jac), ("metric", case.metric)):
        a = np.ascontiguousarray(arr)
        ctx.h2d(getattr(zone, fld), a.ctypes.data, a.nbytes)
    ctx.cv_from_bv()
    ctx.surrogate_init(seed, mech.element_mass_fractions())
    return ctx, zone


def surrogate_bench(args, local):
    """MLP chemistry surrogate against the plain point-implicit integrator on
    the batched H2/air reactors (T ~ U[1000,1600] K, p log-uniform in
    [1,10] atm, phi ~ U[0.5,2], Li-2004, dt = 1e-7 s per step).

    1. training data: the plain work-queue step on `train_cells` reactors for
       `window` steps, one (state, change) row per reactor and step, recorded
       on the device; Adam on the device (tcgen05 forward/backward kernels).
    2. accuracy: unseen reactors, `window` steps from the unburnt state, gated
       surrogate step (default gate, judge every 64th node) vs the plain step:
       ignition delay (time of max dT/dt) and peak temperature, max relative
       error over the reactors that ignite.
    3. throughput: 2^20 unseen reactors advanced `window` steps by the
       surrogate path (judge off: this only builds the run's state mix) and
       then, from that same state, K plain work-queue steps and K gated
       surrogate steps (default gate, judge on), timed with CUDA events.
       Metric: reacting cell-steps/s of each."""
    import torch
    import mechanism
    import surrogate as sg

    mech = mechanism.load("li2004")
    dt, window = 1e-7, args.surrogate_window
    out = {"workload": "constant-volume H2/air reactors, Li-2004 9s/19r, dt 1e-7 s; T~U[1000,1600] K, "
                       "p~logU[1,10] atm, phi~U[0.5,2]", "dtype": "bf16 network, fp32 accumulate; fp64 rest"}
    # 1. training
    n_train = args.surrogate_train_cells
    ctx, _ = _reactor_ctx(mech, cases.reactor_batch(mech, n_train, seed=11), local, 11)
    t0 = time.time()
    X, G = sg.record_trajectories(ctx, n_train, window, dt, torch, device=f"cuda:{local}")
    torch.cuda.synchronize()
    t_rec = time.time() - t0
    t0 = time.time()
    losses = sg.fit(ctx, X, G, epochs=args.surrogate_epochs, batch=8192, lr0=2e-3, lr1=1e-5, seed=3)
    torch.cuda.synchronize()
    t_fit = time.time() - t0
    weights, norm = ctx.surrogate_get_params()
    rows = X.shape[0]
    out["training"] = {"cells": n_train, "steps": window, "rows": rows, "record_s": t_rec, "epochs": args.surrogate_epochs,
                       "train_s": t_fit, "rows_per_s": rows * args.surrogate_epochs / t_fit,
                       "loss_first": losses[0], "loss_last": losses[-1]}
    del X, G
    ctx.close()

    # 2. accuracy on full trajectories
    n_acc = args.surrogate_accuracy_cells
    case = cases.reactor_batch(mech, n_acc, seed=12)
    T0 = case.bv[5, :n_acc].copy()
    traj = {}
    for mode in ("plain", "surrogate"):
        ctx, zone = _reactor_ctx(mech, case, local, 12)
        ctx.surrogate_set_params(weights, norm)
        gate = ctx.surrogate_default_gate()
        stats = []
        Ts = torch.empty((window, n_acc), dtype=torch.float64, device=f"cuda:{local}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for s in range(window):
            if mode == "plain":
                ctx.wu_reaction_step(dt, schedule=1)
            else:
                st = ctx.surrogate_reaction_step(dt, gate, s, want_stats=(s % 50 == 49))
                if st:
                    stats.append(st)
            # temperature plane bv[5] after the step (ngg = 0: plane length = cells)
            ctx.d2d(Ts[s].data_ptr(), zone.bv + 5 * case.P * 8, n_acc * 8)
        e1.record()
        torch.cuda.synchronize()
        traj[mode] = (Ts.cpu().numpy(), e0.elapsed_time(e1), stats)
        ctx.close()
    Tp, Ts_ = traj["plain"][0], traj["surrogate"][0]
    tau_p, pk_p, rise_p = sg.ignition_metrics(dt, T0, Tp)
    tau_s, pk_s, rise_s = sg.ignition_metrics(dt, T0, Ts_)
    ign = (rise_p > 20.0) & (tau_p < (window - 50) * dt)
    st = traj["surrogate"][2]
    out["accuracy"] = {
        "cells": n_acc, "steps": window, "ignited": int(ign.sum()),
        "tau_ign_max_rel_err": float((np.abs(tau_s[ign] - tau_p[ign]) / tau_p[ign]).max()) if ign.any() else None,
        "T_peak_max_rel_err": float((np.abs(pk_s - pk_p) / pk_p).max()),
        "T_max_abs_err_K": float(np.abs(Ts_ - Tp).max()),
        "on_network": sum(x["surrogate"] for x in st) / max(sum(x["cells"] for x in st), 1),
        "plain_ms": traj["plain"][1], "surrogate_ms": traj["surrogate"][1]}
    # the whole window from the unburnt start: total device time of each path
    out["whole_window"] = {"cells": n_acc, "steps": window, "plain_s": traj["plain"][1] * 1e-3,
                           "surrogate_s": traj["surrogate"][1] * 1e-3,
                           "speedup": traj["plain"][1] / traj["surrogate"][1],
                           "note": "includes the per-step copy of the temperature plane for the accuracy check"}

    # 4 (optional). the whole window at a large batch: plain work queue
    # against the gated surrogate from the unburnt start, device time of each
    if args.surrogate_window_cells > 0:
        nw = args.surrogate_window_cells
        case_w = cases.reactor_batch(mech, nw, seed=13)
        ww = {"cells": nw, "steps": window}
        for mode in ("plain", "surrogate"):
            ctx, zone = _reactor_ctx(mech, case_w, local, 13)
            ctx.surrogate_set_params(weights, norm)
            gate = ctx.surrogate_default_gate()
            stats = []
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for s in range(window):
                if mode == "plain":
                    ctx.wu_reaction_step(dt, schedule=1)
                else:
                    st = ctx.surrogate_reaction_step(dt, gate, s, want_stats=(s % 50 == 49))
                    if st:
                        stats.append(st)
            e1.record()
            torch.cuda.synchronize()
            ww[f"{mode}_s"] = e0.elapsed_time(e1) * 1e-3
            if stats:
                ww["on_network"] = sum(x["surrogate"] for x in stats) / sum(x["cells"] for x in stats)
            ctx.close()
        ww["speedup"] = ww["plain_s"] / ww["surrogate_s"]
        out["whole_window_large"] = ww

    # 3. throughput on 2^20 reactors at the run's state mix
    n = args.reacting_cells
    case = cases.reactor_batch(mech, n, seed=2026)
    ctx, zone = _reactor_ctx(mech, case, local, 2026)
    ctx.surrogate_set_params(weights, norm)
    # the advance only builds the state mix that is timed below (judge off)
    adv = ctx.surrogate_default_gate(judge_stride=0)
    t0 = time.time()
    for s in range(window):
        ctx.surrogate_reaction_step(dt, adv, s)
    ctx.sync()
    t_adv = time.time() - t0
    P = case.P
    planes = {"cv": case.param["n_var"], "bv": 6, "sv": case.param["n_scalar"], "reaction_timeScale": 1}
    saved = {k: torch.empty(c * P, dtype=torch.float64, device=f"cuda:{local}") for k, c in planes.items()}
    for k, buf in saved.items():
        ctx.d2d(buf.data_ptr(), getattr(zone, k), buf.numel() * 8)
    k_steps = max(args.steps // 10, 2)
    res = {}
    nsub = torch.zeros(n, dtype=torch.int32, device=f"cuda:{local}")
    for mode in ("plain", "surrogate"):
        for kk, buf in saved.items():
            ctx.d2d(getattr(zone, kk), buf.data_ptr(), buf.numel() * 8)
        gate = ctx.surrogate_default_gate()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stats = []
        e0.record()
        for s in range(k_steps):
            if mode == "plain":
                ctx.wu_reaction_step(dt, schedule=1, nsub_ptr=nsub.data_ptr())
            else:
                stats.append(ctx.surrogate_reaction_step(dt, gate, window + s, want_stats=True))
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        res[mode] = {"cells_per_s": n * k_steps / (ms * 1e-3), "ms_per_step": ms / k_steps, "steps": k_steps}
        if mode == "plain":
            ns_ = nsub.cpu().numpy()
            res[mode].update({"substeps_mean": float(ns_.mean()), "substeps_max": int(ns_.max())})
        else:
            res[mode]["on_network"] = sum(x["surrogate"] for x in stats) / sum(x["cells"] for x in stats)
            res[mode]["last_step"] = stats[-1]
    ctx.close()
    out["throughput"] = {"cells": n, "state": f"after {window} steps ({window * dt * 1e6:.0f} us)",
                         "advance_s": t_adv, **res,
                         "speedup": res["surrogate"]["cells_per_s"] / res["plain"]["cells_per_s"]}
    return out


def _flow_ctx(mech, case, local, seed):
    """A context holding the flow block `case` (mixture, reacting), with the
    start-of-run sequence applied and the surrogate initialised."""
    import corefl_b200 as cfk
    param = dict(case.param)
    param["device"] = local
    ctx = cfk.Context(param, case.faces)
    zone = ctx.alloc_zone(case.mx, case.my, case.mz)
    ctx.set_mechanism(mech)
    for fld, arr in (("bv", case.bv), ("sv", case.sv), ("jac", case.jac), ("metric", case.metric)):
        a = np.ascontiguousarray(arr)
        ctx.h2d(getattr(zone, fld), a.ctypes.data, a.nbytes)
    ctx.properties()
    ctx.boundary_conditions()
    ctx.properties()
    ctx.cv_from_bv()
    ctx.surrogate_init(seed, mech.element_mass_fractions())
    ctx.sync()
    return ctx, zone


def _interior_plane(ctx, zone, case, field, l):
    """Plane l of a padded zone array, interior nodes, as a host array."""
    a = np.empty(case.P)
    ctx.d2h(a.ctypes.data, getattr(zone, field) + l * case.P * 8, case.P * 8)
    return case.interior(a)


def surrogate_flow_bench(args, local):
    """The chemistry surrogate inside the reacting flow step (Wu's splitting
    with the reaction sub-step replaced by the gated network), on reflected-
    shock tubes of stoichiometric H2-O2 with 70 % Ar (PREMIX 9 species / 19
    reactions, WENO5-ch + mixture-averaged viscous fluxes, adiabatic walls).

    1. ignition window (a small tube, Mach 2.6, reflected state ~1400 K): the
       plain run through ignition records one row per node per step
       (cfk_wu_splitting_step_record); the network is trained on the rows; the
       gated surrogate run repeats the window; ignition delay (largest rise of
       the domain's peak T) and peak T of both, fraction of node-steps on the
       network, whole-window device time of each.
    2. the 2048 x 512 tube (wall-normal stretching 1.02, Mach 2.2 incident
       shock into 0.1 atm / 300 K): K plain and K gated surrogate steps from the
       same start with the network of 1.; reacting cell-updates/s of each
       (cells x steps / device time), the reaction sub-step's share, the
       fallback fraction, and the mean T and Y_OH differences after K steps."""
    import torch
    import mechanism
    import surrogate as sg

    mech = mechanism.load("premix_h2_ar")
    dev = f"cuda:{local}"
    out = {"mechanism": "PREMIX H2/O2/Ar 9s/19r", "dtype": "bf16 network, fp32 accumulate; fp64 rest"}
    # 1. ignition window
    nx, ny, W = args.sflow_ign_nx, args.sflow_ign_ny, args.sflow_ign_steps
    small = cases.reflected_shock_tube(mech, nx, ny, length=0.02, height=0.004, mach=2.6)
    n = small.N
    traces, rows = {}, None
    for mode in ("plain", "surrogate", "surrogate_10", "surrogate_all"):
        ctx, zone = _flow_ctx(mech, small, local, 7)
        if mode == "plain":
            X = torch.empty((W * n, sg.cf.SG_NIN), dtype=torch.float32, device=dev)
            G = torch.empty((W * n, sg.cf.SG_NOUT), dtype=torch.float32, device=dev)
        else:
            ctx.surrogate_set_params(weights, norm)
            gate = ctx.surrogate_default_gate(**GATES[mode])
        Tpad = torch.empty(small.P, dtype=torch.float64, device=dev)
        Tint = Tpad.view(small.shape())[small.ngg:small.ngg + 1, small.ngg:small.ngg + ny, small.ngg:small.ngg + nx]
        peak = torch.empty(W, dtype=torch.float64, device=dev)
        t, now, stats = [], 0.0, []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for s_ in range(W):
            if mode == "plain":
                dt = ctx.wu_splitting_step_record(X[s_ * n].data_ptr(), G[s_ * n].data_ptr())
            else:
                dt, st = ctx.wu_splitting_step_surrogate(gate, s_, want_stats=(s_ % 20 == 19))
                if st:
                    stats.append(st)
            now += dt
            t.append(now)
            ctx.d2d(Tpad.data_ptr(), zone.bv + 5 * small.P * 8, small.P * 8)
            peak[s_] = Tint.max()
        e1.record()
        torch.cuda.synchronize()
        traces[mode] = (np.array(t), peak.cpu().numpy(), e0.elapsed_time(e1), stats)
        if mode == "plain":
            t0 = time.time()
            losses = sg.fit(ctx, X, G, epochs=args.sflow_epochs, batch=8192, lr0=2e-3, lr1=1e-5, seed=3)
            torch.cuda.synchronize()
            weights, norm = ctx.surrogate_get_params()
            out["training"] = {"rows": W * n, "epochs": args.sflow_epochs, "train_s": time.time() - t0,
                               "loss_first": losses[0], "loss_last": losses[-1]}
            del X, G
        ctx.close()

    def ignition(tr):
        """Ignition delay (the domain's peak temperature risen by 400 K over its
        value after the first step, interpolated between steps), peak T, and
        the time of the largest single-step rise (reported only: near-equal
        rises of two steps make that argmax flip)."""
        tt, pk = tr[0], tr[1]
        rise = np.diff(np.concatenate([[pk[0]], pk]))
        kr = int(np.argmax(rise))
        t_rise = 0.5 * (tt[kr] + (tt[kr - 1] if kr else 0.0))
        thr = pk[0] + 400.0
        above = np.nonzero(pk > thr)[0]
        if above.size == 0:
            return float("inf"), float(pk.max()), t_rise
        k = int(above[0])
        t0, p0 = (tt[k - 1], pk[k - 1]) if k else (0.0, pk[0])
        return float(t0 + (thr - p0) / (pk[k] - p0) * (tt[k] - t0)), float(pk.max()), t_rise

    tau_p, pk_p, trise_p = ignition(traces["plain"])
    out["ignition_window"] = {
        "case": f"{nx}x{ny} tube 0.02 x 0.004 m, Mach 2.6 incident shock into 0.1 atm / 300 K, {W} steps "
                f"({traces['plain'][0][-1] * 1e6:.1f} us)",
        "tau_ign_plain_s": tau_p, "tau_largest_rise_plain_s": trise_p, "T_peak_plain_K": pk_p,
        "plain_window_ms": traces["plain"][2], "ignition_delay": "peak T risen by 400 K",
        "note": "the plain window includes recording the training rows"}
    for mode in ("surrogate", "surrogate_10", "surrogate_all"):
        tau_s, pk_s, trise_s = ignition(traces[mode])
        out["ignition_window"][mode] = {
            "gate": GATES[mode] or "default", "tau_ign_s": tau_s, "tau_ign_rel_err": abs(tau_s - tau_p) / tau_p,
            "tau_largest_rise_s": trise_s,
            "T_peak_K": pk_s, "T_peak_rel_err": abs(pk_s - pk_p) / pk_p, "window_ms": traces[mode][2],
            **_stat_summary(traces[mode][3])}

    # 2. the 2048 x 512 tube, with a network trained on its own wall strip
    # (the same grid spacing, CFL step and Mach 2.2 states)
    strip = cases.reflected_shock_tube(mech, args.sflow_nx, args.sflow_ny, ny_keep=32)
    weights, norm, train2 = _train_on_flow(mech, strip, local, args.sflow_train_steps, args.sflow_epochs)
    big = cases.reflected_shock_tube(mech, args.sflow_nx, args.sflow_ny)
    K = args.sflow_steps
    r = _plain_vs_surrogate(mech, big, local, weights, norm, K)
    r["training"] = train2
    r["case"] = (f"{big.mx}x{big.my} tube 0.1 x 0.025 m, wall-normal stretching 1.02, Mach 2.2 incident shock "
                 f"into 0.1 atm / 300 K, {K} steps ({r['plain']['simulated_s'] * 1e9:.1f} ns simulated)")
    out["tube_2048x512"] = r
    return out


# gates of the ignition window: the default (few-substeps threshold 50), the
# threshold at 10 substeps, and the rule off
GATES = {"surrogate": {}, "surrogate_10": {"min_substeps": 10.0}, "surrogate_all": {"min_substeps": 0.0}}


def _stat_summary(stats):
    """Fraction of node-steps on the network and the fallback reasons, summed
    over the sampled steps."""
    if not stats:
        return {}
    cells = sum(x["cells"] for x in stats)
    out = {"on_network": sum(x["surrogate"] for x in stats) / max(cells, 1)}
    for k in stats[0]:
        if k.startswith("fallback_") or k in ("judged", "judge_failed"):
            out[k] = sum(x[k] for x in stats) / max(cells, 1)
    return out


def _plain_vs_surrogate(mech, case, local, weights, norm, K, modes=("plain", "surrogate", "surrogate_all")):
    """K Wu-splitting steps of `case` from its initial state with the plain
    point-implicit reaction sub-step and with the gated surrogate (and, with
    "rk3" in modes, K RK3 steps with the explicit chemical source replayed as
    a CUDA graph), each after two untimed steps from a fresh context; device
    time by CUDA events, phase times by the library's profiling; the mean T
    and Y_OH differences of the surrogate run against the plain one."""
    import torch

    res, finals = {}, {}
    oh = mech.index("OH")
    for mode in modes:
        for timed in (False, True):
            ctx, zone = _flow_ctx(mech, case, local, 7)
            ctx.surrogate_set_params(weights, norm)
            gate = ctx.surrogate_default_gate(**GATES.get(mode, {}))
            n = K if timed else 2
            if timed:
                ctx.set_profiling(mode != "rk3")
                ctx.profile_read()
            stats, now = [], 0.0
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            launches0 = ctx.kernel_launches
            e0.record()
            for s_ in range(n):
                if mode == "plain":
                    now += ctx.wu_splitting_step()
                elif mode == "rk3":
                    now += ctx.rk3_step(graph=True)
                else:
                    dt, st_ = ctx.wu_splitting_step_surrogate(gate, s_, want_stats=timed and s_ % 5 == 4)
                    now += dt
                    if st_:
                        stats.append(st_)
            e1.record()
            torch.cuda.synchronize()
            if not timed:
                ctx.close()
                continue
            ms = e0.elapsed_time(e1)
            r = {"cell_updates_per_s": case.N * K / (ms * 1e-3), "ms_per_step": ms / K, "simulated_s": now,
                 "gpu_launches": ctx.kernel_launches - launches0}
            if mode != "rk3":
                ph = ctx.profile_read()
                r["reaction_ms_per_step"] = ph["reaction"][0] / K
                r["phases_ms_per_step"] = {k: v[0] / K for k, v in ph.items()}
            if stats:
                r.update(_stat_summary(stats))
                r["fallback_fraction"] = 1.0 - r["on_network"]
            res[mode] = r
            finals[mode] = (_interior_plane(ctx, zone, case, "bv", 5), _interior_plane(ctx, zone, case, "sv", oh))
            ctx.close()
    Tp, OHp = finals["plain"]
    out = dict(res)
    for mode in modes:
        if not mode.startswith("surrogate"):
            continue
        Ts, OHs = finals[mode]
        out[mode].update({
            "gate": GATES[mode] or "default",
            "speedup_step": res[mode]["cell_updates_per_s"] / res["plain"]["cell_updates_per_s"],
            "speedup_reaction": res["plain"]["reaction_ms_per_step"] / max(res[mode]["reaction_ms_per_step"], 1e-9),
            "mean_T_rel_err": float(abs(Ts.mean() - Tp.mean()) / Tp.mean()),
            "max_T_abs_err_K": float(np.abs(Ts - Tp).max()),
            "mean_Y_OH_abs_err": float(np.abs(OHs - OHp).mean())})
    out["max_Y_OH_plain"] = float(OHp.max())
    return out


def mixing_layer_bench(args, local):
    """The reacting H2/air mixing layer (cases.mixing_layer: air over H2/N2,
    600 K, 1 atm, velocity ratio 1.5, convective Mach 0.2, tanh profile with
    delta_omega 0.5 mm, 1 % white noise at the inflow, WENO7 characteristic +
    mixture-averaged viscous fluxes, Li-2004 9 species / 19 reactions, span
    periodic).  The network is trained on rows recorded from plain
    Wu-splitting steps of a small block of the same layer; then the
    nx x ny x nz block runs K steps each of plain Wu splitting, Wu splitting
    with the gated surrogate, and RK3 with the explicit chemical source as a
    CUDA graph: reacting cell-updates/s, fallback fraction, and the mean T
    and Y_OH differences of the surrogate run against the plain run."""
    import torch
    import mechanism
    import surrogate as sg

    mech = mechanism.load("li2004")
    # a 64 x 32 x 16 piece of the same grid (the same spacing and CFL step)
    small = cases.mixing_layer(mech, args.ml_nx, args.ml_ny, args.ml_nz, window=(64, 32, 16))
    weights, norm, train = _train_on_flow(mech, small, local, args.ml_train_steps, args.sflow_epochs)
    big = cases.mixing_layer(mech, args.ml_nx, args.ml_ny, args.ml_nz)
    K = args.ml_steps
    r = _plain_vs_surrogate(mech, big, local, weights, norm, K, modes=("plain", "surrogate", "surrogate_all", "rk3"))
    r["case"] = (f"{big.mx}x{big.my}x{big.mz} mixing layer 0.05 x 0.025 x 0.0125 m (y clustered), {K} steps "
                 f"({r['plain']['simulated_s'] * 1e9:.1f} ns simulated)")
    r["training"] = train
    return r


def _train_on_flow(mech, case, local, steps, epochs):
    """Training rows from `steps` plain Wu steps of `case` (one per node and
    step, cfk_wu_splitting_step_record), then Adam on the device; returns the
    weights, the standardisation and a summary."""
    import torch
    import surrogate as sg

    dev = f"cuda:{local}"
    n = case.N
    ctx, _ = _flow_ctx(mech, case, local, 9)
    X = torch.empty((steps * n, sg.cf.SG_NIN), dtype=torch.float32, device=dev)
    G = torch.empty((steps * n, sg.cf.SG_NOUT), dtype=torch.float32, device=dev)
    for s_ in range(steps):
        ctx.wu_splitting_step_record(X[s_ * n].data_ptr(), G[s_ * n].data_ptr())
    t0 = time.time()
    losses = sg.fit(ctx, X, G, epochs=epochs, batch=8192, lr0=2e-3, lr1=1e-5, seed=3)
    torch.cuda.synchronize()
    weights, norm = ctx.surrogate_get_params()
    ctx.close()
    return weights, norm, {"case": f"{case.mx}x{case.my}x{case.mz} piece of the same grid", "rows": steps * n,
                           "epochs": epochs, "train_s": time.time() - t0, "loss_first": losses[0],
                           "loss_last": losses[-1]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", "--block-n", dest="n", type=int, default=N_NODES, help="nodes per direction (default 257)")
    ap.add_argument("--scheme", type=int, default=72,
                    help="inviscid_scheme: 72/52 WENO7/5 characteristic (default 72), 1 LF, 2 Roe, 3 AUSM+, 4 HLLC")
    ap.add_argument("--reconstruction", type=int, default=2, help="for schemes 1-4: 1 first order, 2 MUSCL, 3 NND2")
    ap.add_argument("--e2e-steps", type=int, default=None, help="steps of the end-to-end measurement (default: --steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default WENO tile shapes")
    ap.add_argument("--no-reacting", action="store_true")
    ap.add_argument("--reacting-only", action="store_true", help="only the batched-reactor measurement")
    ap.add_argument("--reacting-cells", type=int, default=1 << 20)
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--surrogate-only", action="store_true", help="only the MLP surrogate measurement")
    ap.add_argument("--surrogate-window", type=int, default=600, help="steps of the training/accuracy window")
    ap.add_argument("--surrogate-train-cells", type=int, default=16384)
    ap.add_argument("--surrogate-accuracy-cells", type=int, default=16384)
    ap.add_argument("--surrogate-epochs", type=int, default=200)
    ap.add_argument("--surrogate-window-cells", type=int, default=0,
                    help="also time the whole window at this many reactors, plain against surrogate (0: off)")
    ap.add_argument("--no-surrogate-flow", action="store_true")
    ap.add_argument("--surrogate-flow-only", action="store_true", help="only the surrogate-in-the-flow measurement")
    ap.add_argument("--sflow-nx", type=int, default=2048)
    ap.add_argument("--sflow-ny", type=int, default=512)
    ap.add_argument("--sflow-steps", type=int, default=100, help="timed Wu steps of the 2048x512 tube per mode")
    ap.add_argument("--sflow-ign-nx", type=int, default=128)
    ap.add_argument("--sflow-ign-ny", type=int, default=16)
    ap.add_argument("--sflow-ign-steps", type=int, default=600)
    ap.add_argument("--sflow-epochs", type=int, default=300)
    ap.add_argument("--sflow-train-steps", type=int, default=100, help="recorded Wu steps of the tube's wall strip")
    ap.add_argument("--no-mixing-layer", action="store_true")
    ap.add_argument("--mixing-layer-only", action="store_true", help="only the reacting mixing-layer measurement")
    ap.add_argument("--ml-nx", type=int, default=512)
    ap.add_argument("--ml-ny", type=int, default=256)
    ap.add_argument("--ml-nz", type=int, default=128)
    ap.add_argument("--ml-steps", type=int, default=10, help="timed steps of the mixing layer per mode")
    ap.add_argument("--ml-train-steps", type=int, default=100)
    args = ap.parse_args()
    rank, world, local = _env_rank()
    args.warmup = max(args.warmup, 3)
    if args.e2e_steps is None:
        args.e2e_steps = args.steps

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import corefl_b200 as cfk

    if args.reacting_only:
        torch.cuda.set_device(local)
        print(json.dumps({"reacting": reacting_bench(args, local, 1, None)}), flush=True)
        return
    if args.surrogate_only:
        torch.cuda.set_device(local)
        print(json.dumps({"surrogate": surrogate_bench(args, local)}), flush=True)
        return
    if args.surrogate_flow_only:
        torch.cuda.set_device(local)
        print(json.dumps({"surrogate_flow": surrogate_flow_bench(args, local)}), flush=True)
        return
    if args.mixing_layer_only:
        torch.cuda.set_device(local)
        print(json.dumps({"mixing_layer": mixing_layer_bench(args, local)}), flush=True)
        return

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{local}"))
    else:
        torch.cuda.set_device(0)

    n = args.n
    case = cases.sine_wave(n=n, scheme=args.scheme, viscous=True, cfl=0.5, reconstruction=args.reconstruction)
    param = dict(case.param)
    param["device"] = local
    ctx = cfk.Context(param, case.faces)
    zone = ctx.alloc_zone(case.mx, case.my, case.mz)
    _upload(ctx, zone, case)
    ctx.properties()
    ctx.boundary_conditions()
    ctx.properties()
    ctx.cv_from_bv()
    ctx.sync()
    # tile shapes of the WENO sweeps, timed on this block (outside the timed region)
    tiles, tile_ms = ([0, 0, 0], None) if args.no_autotune else ctx.autotune_tiles(reps=3)
    visc_var, visc_ms = ctx.viscous_variant()

    for _ in range(args.warmup):
        ctx.rk3_step(want_dt=False)
    ctx.sync()

    # ---- timed region: K plain steps, phase events on the launching stream
    ctx.set_profiling(True)
    ctx.profile_read()  # clear
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = ctx.kernel_launches
    with ClockSampler(local) as clk:
        start.record()
        for _ in range(args.steps):
            ctx.rk3_step(want_dt=False)
        stop.record()
        torch.cuda.synchronize()
    ms = start.elapsed_time(stop)
    launches = ctx.kernel_launches - launches0
    phases = ctx.profile_read()
    ctx.set_profiling(False)
    ms = max_over_ranks(ms, dist, f"cuda:{local}")
    if dist:
        dist.barrier()
    nodes = case.N
    value = nodes * args.steps * world / (ms * 1e-3)

    # ---- roofline of the dominant kernel (the three inviscid sweeps)
    inv_ms, inv_k = phases["inviscid"]
    faces_per_launch = ((case.mx + 1) * case.my * case.mz + case.mx * (case.my + 1) * case.mz +
                        case.mx * case.my * (case.mz + 1)) / 3.0
    avg_launch_ms = inv_ms / max(inv_k, 1)
    hbm_peak = None
    mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(mp):
        with open(mp) as f:
            hbm_peak = json.load(f).get("hbm_gbs")
    if args.scheme == 72:
        achieved = FLOPS_PER_FACE_WENO7_CH * faces_per_launch / (avg_launch_ms * 1e-3) / 1e12
        peak = cfk.measure_fp64_peak()
        traffic, traffic_source = weno_traffic_per_launch(case.mx * case.my * case.mz)
        roofline = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                    "traffic": traffic, "traffic_source": traffic_source,
                    "kernel": "weno_air_flux_diff<dir,7> (x/y/z sweeps)",
                    "peak_source": "measured live: cfk_measure_fp64_peak FMA-chain kernel",
                    "avg_launch_ms": avg_launch_ms, "flops_per_launch": FLOPS_PER_FACE_WENO7_CH * faces_per_launch,
                    "flops_source": "ncu DFMA/DADD/DMUL counters per face, 161^3 "
                                    "(profiles/weno_air_flux_diff_161_fp64_counts.md)",
                    "frac_hand_count": FLOPS_PER_FACE_WENO7_CH_HAND * faces_per_launch / (avg_launch_ms * 1e-3)
                    / 1e12 / peak}
    else:
        # primitive-variable schemes are HBM-bound: algorithmic bytes per node
        # and direction = bv[5] + metric[3] + jac + dq[5] read-modify-write
        # (Roe: + the six other metric terms of the entropy-fix width)
        per_node = 8 * (5 + 3 + 1 + 10 + (6 if args.scheme == 2 else 0))
        achieved = per_node * case.N / (avg_launch_ms * 1e-3) / 1e9
        peak = hbm_peak
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak if peak else None, "traffic": None,
                    "kernel": f"pv_air_flux_diff<dir,{args.scheme},{args.reconstruction}> (x/y/z sweeps)",
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs", "avg_launch_ms": avg_launch_ms,
                    "bytes_per_launch": per_node * case.N}

    # ---- end to end through the C ABI with pinned host buffers.  Each step
    # uploads its input (bv, 6 planes) from pinned host memory and reads its
    # result (cv, 5 planes) back.  The copies run on their own streams and
    # copy engines, double-buffered through device staging arrays, so that
    # step k+1's upload and step k-1's download overlap step k's compute:
    #   h2d stream:     H2D bv_host -> stage_in[k % 2]
    #   compute stream: D2D stage_in -> zone.bv, cv_from_bv, rk3_step,
    #                   D2D zone.cv -> stage_out[k % 2]
    #   d2h stream:     D2H stage_out[k % 2] -> cv_host
    P = case.P
    h2d_bytes = 6 * P * 8
    d2h_bytes = 5 * P * 8
    hb_ptr, hc_ptr = ctypes.c_void_p(), ctypes.c_void_p()
    L = cfk.lib()
    assert L.cfk_host_alloc(h2d_bytes, ctypes.byref(hb_ptr)) == 0
    assert L.cfk_host_alloc(d2h_bytes, ctypes.byref(hc_ptr)) == 0
    ctypes.memmove(hb_ptr, np.ascontiguousarray(case.bv).ctypes.data, h2d_bytes)
    dev = torch.device(f"cuda:{local}")
    stage_in = [torch.empty(6 * P, dtype=torch.float64, device=dev) for _ in range(2)]
    stage_out = [torch.empty(5 * P, dtype=torch.float64, device=dev) for _ in range(2)]
    s_comp, s_up, s_down = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    h_comp, h_up, h_down = (ctypes.c_void_p(s.cuda_stream) for s in (s_comp, s_up, s_down))
    ev = lambda: torch.cuda.Event()
    up_done, in_free, out_ready, out_free = ([ev() for _ in range(2)] for _ in range(4))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.sync()
    torch.cuda.synchronize()
    e0.record(s_comp)
    s_up.wait_event(e0)
    s_down.wait_event(e0)
    for k in range(args.e2e_steps):
        b = k % 2
        if k >= 2:
            s_up.wait_event(in_free[b])
        ctx.h2d(stage_in[b].data_ptr(), hb_ptr, h2d_bytes, h_up)
        up_done[b].record(s_up)
        s_comp.wait_event(up_done[b])
        ctx.d2d(zone.bv, stage_in[b].data_ptr(), h2d_bytes, h_comp)
        in_free[b].record(s_comp)
        ctx.cv_from_bv(h_comp)
        ctx.rk3_step(h_comp, want_dt=False)
        if k >= 2:
            s_comp.wait_event(out_free[b])
        ctx.d2d(stage_out[b].data_ptr(), zone.cv, d2h_bytes, h_comp)
        out_ready[b].record(s_comp)
        s_down.wait_event(out_ready[b])
        ctx.d2h(hc_ptr, stage_out[b].data_ptr(), d2h_bytes, h_down)
        out_free[b].record(s_down)
    s_comp.wait_stream(s_down)
    e1.record(s_comp)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1)
    ms_e2e = max_over_ranks(ms_e2e, dist, f"cuda:{local}")
    e2e = {"value": nodes * args.e2e_steps * world / (ms_e2e * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes, "steps": args.e2e_steps,
           "ms_per_step": ms_e2e / args.e2e_steps,
           "path": "cfk_memcpy_h2d(bv, pinned) + cfk_memcpy_d2d + cfk_compute_cv_from_bv + cfk_rk3_step + "
                   "cfk_memcpy_d2d + cfk_memcpy_d2h(cv, pinned); copies on their own streams, double-buffered, "
                   "overlapping the neighbouring steps' compute"}
    L.cfk_host_free(hb_ptr)
    L.cfk_host_free(hc_ptr)
    ctx.close()

    reacting = None if args.no_reacting else reacting_bench(args, local, world, dist)
    # the surrogate and reacting-flow measurements are one GPU's work: they run
    # in single-GPU runs only, so that a multi-GPU run does not hold every GPU
    # while one rank works through them
    single = world == 1
    surrogate = None if (args.no_surrogate or args.no_reacting or not single) else surrogate_bench(args, local)
    surrogate_flow = (None if (args.no_surrogate_flow or args.no_reacting or not single)
                      else surrogate_flow_bench(args, local))
    mixing_layer = (None if (args.no_mixing_layer or args.no_reacting or not single)
                    else mixing_layer_bench(args, local))

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:  # the CPU baseline is a single-GPU run's figure
            cpu = cpu_baseline_sample(args.scheme, args.reconstruction, case=case)
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "3-D viscous sine wave, curvilinear periodic block, "
                                   + ("WENO7-ch" if args.scheme == 72 else f"inviscid_scheme {args.scheme} "
                                      f"reconstruction {args.reconstruction}") +
                                   " + 2nd-order viscous, SSP-RK3 CFL 0.5 (device dt)",
                       "nodes": f"{n}^3", "global_nodes": nodes * world,
                       "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (cv alone "
                       f"{5 * P * 8 / 1e6:.0f} MB)", "weno_tile_variants": tiles, "autotune_ms": tile_ms,
                       "viscous_form": ["staged", "ring", "ring + L2 prefetch of the metric"][visc_var], "viscous_form_ms": visc_ms},
            "phases_ms_per_step": {k: v[0] / args.steps for k, v in phases.items()},
            "gpu_launches": launches,
            "roofline": roofline,
            "hbm_peak_gbs": hbm_peak,
            "cpu_baseline": cpu,
            "reference_gpu": dict(REFERENCE_GPU_257) if (n == N_NODES and args.scheme == 72) else None,
            "e2e": e2e,
            "clocks": clk.summary(),
            "reacting": reacting,
            "surrogate": surrogate,
            "surrogate_flow": surrogate_flow,
            "mixing_layer": mixing_layer,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
