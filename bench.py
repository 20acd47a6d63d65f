#!/usr/bin/env python
"""Throughput of Canard's full time step on B200, in Mpoint-steps/s.

Workload (default): Taylor-Green vortex on a single 256^3-cell block (257^3
stored points, the reference's point count including the periodic shared
points), viscous, FP64, the full reference time step: 15 compact filter
passes, then 4 Runge-Kutta stages (primitives, viscous stresses, fluxes, 27
compact line solves per stage, GCBC/sponge where present, RK update, junction
averaging), with the reference's dt schedule. Synthetic, seeded input.

The headline runs the fast FP64 mode (every value FP64; split line solves
with FMA, held to 1e-10 relative L2 of the oracle after 10 steps); the
bit-exact FP64 path and FP32-mixed are timed beside it on the same workload
(`--precision fp64|fast|fp32` picks the headline).

One step = one call of the reference's time-loop body. `value` is device time
(CUDA events on the launching stream, max over ranks) with the state resident
in HBM; `e2e` goes through the public C ABI with the state in pinned host
memory copied in and out every step. Multi-GPU runs are independent replicas
(the single-block case has no partition on this path), so scaling is weak.

`--impl reference` times the reference algorithm on the host CPU cores (the
oracle restatement: the Fortran reference cannot be compiled in this image)
on the same workload, --warmup untimed and --steps timed full steps.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# the headline metric: Mpoint-steps/s of the plain FP64 path, with the
# FP32-mixed and batched forms beside it and the dominant kernel's HBM GB/s
METRIC = "Mpoint-steps/s on 1 B200: FP32-mixed/batched vs FP64 plain; HBM GB/s vs peak"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=256, help="cells per direction of the TGV block")
    p.add_argument("--config", default="tgv", choices=["tgv", "batched", "curv4", "vortex"],
                   help="tgv: single TGV block (default); batched: 64 independent cases with sides "
                        "in 32..96; curv4: 4-block curvilinear grid with GCBC and sponge; vortex: "
                        "isentropic vortex through a GCBC outflow")
    p.add_argument("--precision", default="fast", choices=["fp64", "fast", "fp32"],
                   help="fp64: plain FP64 path (bit-exact with the oracle); fast: FP64 throughout with the split "
                        "line solves and FMA (within 1e-10 of the oracle); fp32: FP32 line solves, fluxes, "
                        "viscous stresses and GCBC with the FP64 state, RK update, metrics and LU factors")
    p.add_argument("--acc-nx", type=int, default=384)
    p.add_argument("--acc-ny", type=int, default=256)
    p.add_argument("--acc-nz", type=int, default=128)
    p.add_argument("--cpu-steps", type=int, default=5)
    p.add_argument("--e2e-steps", type=int, default=10,
                   help="steps of the end-to-end measurement through host memory (one canard_step_host call: "
                        "the first step's copy in and the last one's copy out are not overlapped)")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--mode", default="step", choices=["step", "kernels", "accuracy", "cpu"],
                   help="step: the time-step benchmark (default); kernels: isolated derivative and filter "
                        "launches per direction on 5 noise fields, checked against the oracle; accuracy: "
                        "FP32-mixed against FP64 on the vortex case after 50/200/1000 steps; cpu: the oracle "
                        "(CPU restatement of the reference) on --config, --cpu-steps steps after one warm-up "
                        "step, with --cpu-threads threads")
    p.add_argument("--cpu-threads", type=int, default=0, help="oracle threads (0: all host threads)")
    p.add_argument("--no-autotune", action="store_true",
                   help="skip the line-tile autotuner (by default every timed context is tuned first; the "
                        "per-case baseline of the batched comparison never is)")
    p.add_argument("--tune-file", default="",
                   help="line-kernel choices of the timed context: read from this JSON file when it exists "
                        "(no autotuning), else autotuned and written to it, so that a second run (a profiler's "
                        "launch list, for one) launches the same kernels")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the FP32-mixed and batched comparison lines added to the default run")
    return p.parse_args()


def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def state_errors(qg, qr, uref):
    """Relative L2 error per conserved variable of qg against qr; momentum
    components against the momentum scale ||rho|| * uref where that exceeds
    their own norm (a component that is zero by symmetry has no relative error)."""
    rho = np.linalg.norm(qr[0].ravel())
    out = []
    for v in range(5):
        den = np.linalg.norm(qr[v].ravel())
        if 1 <= v <= 3:
            den = max(den, rho * uref)
        out.append(float(np.linalg.norm((qg[v] - qr[v]).ravel()) / den))
    return out


def time_steps(ctx, steps, stream, torch):
    """Device milliseconds of `steps` steps (CUDA events on the launching stream)."""
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    ctx.step(steps)
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def tune_context(ctx, args):
    """The timed context's line kernels: autotuned (the default), read from
    --tune-file when that exists, or none (--no-autotune)."""
    if args.no_autotune:
        return None
    if args.tune_file and os.path.exists(args.tune_file):
        with open(args.tune_file) as f:
            tuning = json.load(f)
        for t in tuning:
            ch = t["chunks"] if isinstance(t["chunks"], int) else 0
            ctx.set_line_kind(t["group"], t["dir"], t["kind"], ch)
        return tuning
    tuning = ctx.autotune(reps=3)
    if args.tune_file:
        with open(args.tune_file, "w") as f:
            json.dump(tuning, f)
    return tuning


def precision_extra(args, api, cases, torch, stream, prec):
    """Another precision on the same workload: its throughput (autotuned as the
    headline), and the error after 10 steps from the initial condition against
    the bit-exact FP64 path."""
    cs = cases.tgv(args.n)
    c = api.Context(cs, precision=prec)
    if not args.no_autotune:
        c.autotune(reps=3)
    c.set_stream(stream.cuda_stream)
    c.step(args.warmup)
    ms = time_steps(c, args.steps, stream, torch)
    c.close()
    v = cs.npts * args.steps / (ms / 1e3) / 1e6
    out = {"value": v, "unit": "Mpoint-steps/s", "ms_per_step": ms / args.steps, "steps": args.steps}
    if prec != api.FP64:
        a = api.Context(cs)
        b = api.Context(cs, precision=prec)
        a.step(10)
        b.step(10)
        out["rel_l2_vs_fp64_bit_exact_after_10_steps"] = state_errors(b.state(0), a.state(0), 0.1)
        out["note"] = ("per variable (rho, rho u, rho v, rho w, rho E); momenta against ||rho|| * 0.1 (TGV V0) "
                       "where that exceeds their own norm")
        a.close()
        b.close()
    return out


def batched_extra(args, api, cases, torch, stream):
    """64 independent cases (sides 32..96): one context, one launch per phase
    and direction for all cases, each step one CUDA graph, FP32-mixed and
    FP64; against the per-case FP64 plain path (one context per case, case
    after case: kernels launched one by one, and with each case's own step
    graph)."""
    allc = cases.batched(64, seed=11)
    npts = sum(c.npts for c in allc)
    out = {"workload": "64 cases, sides 32..96 (seed 11), TGV / periodic vortex, Mach 0.1-0.5, Re 400-3200",
           "points": npts, "steps": args.steps}
    states = {}
    gaps = {}
    for key, prec in (("fp32_mixed_graph", api.FP32_MIXED), ("fp64_graph", api.FP64)):
        g = api.Context(allc, precision=prec)
        if not args.no_autotune:
            g.autotune(reps=3)
        g.set_stream(stream.cuda_stream)
        g.step(args.warmup)
        ms = time_steps(g, args.steps, stream, torch)
        out[key] = npts * args.steps / (ms / 1e3) / 1e6
        states[key] = [g.state(0, i) for i in range(len(allc))]
        # the step's kernels alone (each bracketed by CUDA events, launched one
        # by one) against the graph's step: what launch gaps and kernel tails
        # cost, the most a persistent kernel per stage could take back without
        # fusing work
        g.set_timers(True)
        g.step(1)
        kms = sum(f["ms"] for f in g.timers().values())
        g.set_timers(False)
        gaps[key] = {"graph_ms_per_step": ms / args.steps, "kernels_ms_per_step": kms,
                     "outside_kernels_fraction": max(0.0, 1.0 - kms / (ms / args.steps))}
        g.close()
    out["graph_vs_kernel_time"] = gaps
    ctxs = []
    for c in allc:
        x = api.Context(c)
        x.set_graphs(False)
        x.set_stream(stream.cuda_stream)
        x.step(args.warmup)
        ctxs.append(x)
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    a.record(stream)
    for x in ctxs:
        x.step(args.steps)
    b.record(stream)
    torch.cuda.synchronize()
    ms = max(a.elapsed_time(b), (time.perf_counter() - t0) * 1e3)
    out["fp64_per_case_plain"] = npts * args.steps / (ms / 1e3) / 1e6
    ref = [x.state(0) for x in ctxs]
    # the same per-case contexts with their own step graphs on (one graph
    # launch per case and step)
    for x in ctxs:
        x.set_graphs(True)
        x.step(1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    a.record(stream)
    for x in ctxs:
        x.step(args.steps)
    b.record(stream)
    torch.cuda.synchronize()
    ms = max(a.elapsed_time(b), (time.perf_counter() - t0) * 1e3)
    out["fp64_per_case_graphs"] = npts * args.steps / (ms / 1e3) / 1e6
    for x in ctxs:
        x.close()
    out["speedup_fp32_graph_vs_fp64_per_case"] = out["fp32_mixed_graph"] / out["fp64_per_case_plain"]
    out["speedup_fp64_graph_vs_fp64_per_case"] = out["fp64_graph"] / out["fp64_per_case_plain"]
    out["speedup_fp32_graph_vs_fp64_per_case_graphs"] = out["fp32_mixed_graph"] / out["fp64_per_case_graphs"]
    out["fp64_graph_bit_identical_to_per_case"] = bool(all(np.array_equal(s, r)
                                                            for s, r in zip(states["fp64_graph"], ref)))
    errs = [state_errors(s, r, 0.5) for s, r in zip(states["fp32_mixed_graph"], ref)]
    out["fp32_max_rel_l2_vs_fp64"] = float(max(max(e) for e in errs))
    out["fp32_max_abs_vs_fp64"] = float(max(np.abs(s - r).max() for s, r in zip(states["fp32_mixed_graph"], ref)))
    return out


def workload_cases(args, cases, world=1, rank=0):
    """The timed cases of this rank, all cases of the job and the workload's
    description (one for both arms, so that the reference arm runs the same
    config)."""
    if args.config == "tgv":
        case_list = all_cases = [cases.tgv(args.n)]
        workload = (f"tgv{args.n}: Taylor-Green vortex {args.n}^3 cells ({args.n + 1}^3 points), Re 1600, "
                    "Mach 0.1, viscous, FP64 plain, full time step")
    elif args.config == "batched":
        from canard_b200 import shard
        all_cases = cases.batched(64, seed=11)
        mine = shard.my_cases([c.npts for c in all_cases], world, rank)
        case_list = [all_cases[i] for i in mine]
        workload = ("batched: 64 independent single-block cases (sides 32..96, TGV / periodic vortex, "
                    "Mach 0.1-0.5, Re 400-3200), FP64, one launch per phase and direction for all cases"
                    + (f", sharded over {world} ranks by point count" if world > 1 else ""))
    elif args.config == "curv4":
        case_list = all_cases = [cases.curvilinear_4block()]
        workload = "curv4: 4 blocks of 192x128x64 cells, curvilinear, GCBC in/outflow, sponge, Re 1e5, FP64"
    else:
        case_list = all_cases = [cases.vortex()]
        workload = "vortex: 384x256x128 cells, isentropic vortex, GCBC outflow, FP64"
    if args.precision == "fp32":
        workload = workload.replace("FP64 plain", "FP32-mixed").replace(", FP64", ", FP32-mixed")
    elif args.precision == "fast":
        workload = workload.replace("FP64 plain", "FP64").replace(", FP64", ", FP64")
    return case_list, all_cases, workload


def config_dict(args, workload, ncases, job_points, npts, world):
    """The bench line's config, the same for the device arm and the reference arm."""
    mode = {"fp64": "FP64, bit-exact with the reference's operation order",
            "fast": "FP64 fast mode (split and two-ended line solves with FMA; within 1e-10 of the reference "
                    "after 10 steps)",
            "fp32": "FP32-mixed (FP32 line solves and fluxes; FP64 state, RK update, metrics and LU)"}[args.precision]
    return {"workload": workload, "cases": ncases, "points": job_points, "precision": args.precision,
            "arithmetic": mode,
            "l2": "inputs larger than L2 (state, metrics and work fields ~"
                  f"{(54 * 8 + (41 * 4 if args.precision == 'fp32' else 0)) * npts / 1e9:.1f} GB resident on the "
                  "device; larger than the host caches on the CPU arm too)",
            "parallelism": ("case shards" if args.config == "batched" else "replicas") if world > 1 else "single"}


def oracle_rate(case_list, steps, warmup, threads):
    """The oracle (CPU restatement of the reference) over the cases, one after
    the other: Mpoint-steps/s of `steps` timed steps after `warmup` untimed
    ones, and the timed seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    npts, secs = 0, 0.0
    for cs in case_list:
        o = po.Oracle(cs, threads=threads)
        if warmup:
            o.step(warmup)
        t0 = time.perf_counter()
        o.step(steps)
        secs += time.perf_counter() - t0
        npts += cs.npts
        del o
    return npts * steps / secs / 1e6, secs


def config_cases(args, cases):
    if args.config == "tgv":
        return [cases.tgv(args.n)], f"tgv{args.n}"
    if args.config == "batched":
        return cases.batched(64, seed=11), "batched64"
    if args.config == "curv4":
        return [cases.curvilinear_4block()], "curv4"
    return [cases.vortex()], "vortex"


def cpu_mode(args):
    """The oracle on a whole config: Mpoint-steps/s over --cpu-steps steps
    (after one untimed step); batched cases run one after the other."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from canard_b200 import cases
    threads = args.cpu_threads or (os.cpu_count() or 1)
    case_list, name = config_cases(args, cases)
    npts, secs = 0, 0.0
    for cs in case_list:
        o = po.Oracle(cs, threads=threads)
        o.step(1)
        t0 = time.perf_counter()
        o.step(args.cpu_steps)
        secs += time.perf_counter() - t0
        npts += cs.npts
        del o
    v = npts * args.cpu_steps / secs / 1e6
    return {"mode": "cpu", "config": name, "points": npts, "steps": args.cpu_steps, "threads": threads,
            "seconds": secs, "value": v, "unit": "Mpoint-steps/s", "kind": "port (C++ restatement of the reference)"}


def kernels_mode(args, api, cases, torch):
    """Isolated line solves (the reference's deriv / filte over one direction):
    5 FP64 fields of seeded N(0,1) noise plus sin modes k = 1..32 on the TGV
    block; per (precision, operation, direction) the average device time of
    one launch over the 5 fields, its algorithmic GB/s (each field read and
    written once) against the measured copy peak, and the error against the
    oracle's line solve of the same fields."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    cs = cases.tgv(args.n)
    blk = cs.blocks[0]
    fields = cases.noise_fields(blk, 5)
    o = po.Oracle(cs, setup=False, threads=os.cpu_count() or 1)
    ref = {}
    for op in (0, 1):
        for nn in (1, 2, 3):
            res = []
            for k in range(5):
                f = fields[k].ravel().copy()
                if op == 0:
                    o.mpigo([f.copy()], 0, 1, 0, k + 1, k + 1)
                    r = np.zeros_like(f)
                    o.deriv(0, f, r, nn, k + 1)
                else:
                    o.mpigo([f], 1, 1, 0, k + 1, k + 1)
                    o.filte(0, f, {2: 1, 3: 2, 1: 3}[nn], k + 1)
                    r = f
                res.append(r.reshape(blk.shape))
            ref[(op, nn)] = np.stack(res)
        o = po.Oracle(cs, setup=False, threads=os.cpu_count() or 1)  # fresh filter send chain
    peak, peak_kind = peaks()
    rows = []
    # fp64-tmem: the FP64 eta/zeta kernel that keeps the elimination results in
    # tensor memory (an autotuner candidate), pinned for the comparison
    # fp32-stream: the mixed filter that streams the FP64 state into FP32
    # right-hand sides (an autotuner candidate), pinned for the comparison
    for prec, name in ((api.FP64, "fp64"), (api.FP64, "fp64-tmem"), (api.FP64_FAST, "fp64-fast"),
                       (api.FP64_FAST, "fp64-quad"), (api.FP32_MIXED, "fp32"), (api.FP32_MIXED, "fp32-quad"),
                       (api.FP32_MIXED, "fp32-stream"), (api.FP64_FAST, "fp64-twist"), (api.FP32_MIXED, "fp32-twist")):
        ctx = api.Context(cs, precision=prec, setup=False, upload_state=False)
        for op in (0, 1):
            if (name == "fp32-stream" and op == 0) or (name.endswith("quad") and op == 1):
                continue
            for nn in (1, 2, 3):
                if name == "fp64-tmem" and nn > 1:
                    ctx.set_line_kind("flux" if op == 0 else "filter", "xi eta zeta".split()[nn - 1], "fp64-tmem")
                if name == "fp32-stream":
                    ctx.set_line_kind("filter", "xi eta zeta".split()[nn - 1], "fp64-stream/fp32-split")
                if name.endswith("quad"):
                    ctx.set_line_kind("flux", "xi eta zeta".split()[nn - 1], name)
                if name.endswith("twist"):  # two-ended solve (two warps per 32 lines)
                    kt = name if (op == 0 or name == "fp64-twist") else "fp64-tile/fp32-twist"
                    ctx.set_line_kind("flux" if op == 0 else "filter", "xi eta zeta".split()[nn - 1], kt)
                # xi runs on the shared-memory tiles here too: the filter's interface calls
                # advance the send chains of all directions in the oracle's order
                out, ms = ctx.line_bench(op, nn, fields, reps=args.steps)
                if name == "fp64-tmem" and nn == 1:
                    continue
                es = 4 if (name in ("fp32", "fp32-quad", "fp32-twist") and op == 0) else 8
                gbs = 5 * blk.npts * 2 * es / (ms / 1e3) / 1e9
                r = ref[(op, nn)]
                err = float(np.linalg.norm((out - r).ravel()) / np.linalg.norm(r.ravel()))
                rows.append({"precision": name, "op": "deriv" if op == 0 else "filter", "dir": "xi eta zeta".split()[nn - 1],
                             "ms_per_launch": ms, "gbs": gbs, "frac_of_peak": gbs / peak,
                             "rel_l2_vs_oracle": err, "bit_exact": bool(np.array_equal(out, r))})
            # the filter chain of a context carries over calls: a fresh context per operation
        ctx.close()
    return {"mode": "kernels", "workload": f"tgv{args.n} block ({args.n + 1}^3 points), 5 fields of N(0,1) noise "
            "+ sum of sin modes k=1..32 (seed 20261203)", "peak_gbs": peak, "peak_kind": peak_kind,
            "launches_timed": args.steps, "kernels": rows}


def accuracy_mode(args, api, cases, torch):
    """The C4 study: the isentropic vortex through a GCBC outflow.

    * The 384x256x128 case on the GPU after 50 ... 1000 steps: FP32-mixed and
      the fast FP64 mode against the bit-exact FP64 path (relative L2 per
      conserved variable, momenta against ||rho|| * 0.5), and whether each
      state is still finite.
    * A 96x64x32 copy against the oracle after 50, 200 and 1000 steps, in all
      three precisions (the oracle's 1000 steps take a few minutes on the
      host cores)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    out = {"mode": "accuracy"}
    big = cases.vortex(nx=args.acc_nx, ny=args.acc_ny, nz=args.acc_nz)
    ctxs = {"fp64": api.Context(big), "fast": api.Context(big, precision=api.FP64_FAST),
            "fp32": api.Context(big, precision=api.FP32_MIXED)}
    done, rows = 0, []
    stopped = {}

    def advance(ctx, key, k):
        # the dt reduction raises the overflow error once a state is non-finite
        if key in stopped:
            return
        try:
            ctx.step(k)
        except api.CanardError as e:
            stopped[key] = f"stopped between steps {done} and {done + k}: {e}"

    for n in (50, 100, 200, 400, 1000):
        for key, ctx in ctxs.items():
            advance(ctx, key, n - done)
        q = {key: ctx.state(0) for key, ctx in ctxs.items()}
        done = n
        row = {"steps": n, "time": ctxs["fp64"].time()[5]}
        for key in ctxs:
            row[f"{key}_finite"] = key not in stopped and bool(np.isfinite(q[key]).all())
        for key in ("fast", "fp32"):
            if row["fp64_finite"] and row[f"{key}_finite"]:
                row[f"rel_l2_{key}_vs_fp64"] = state_errors(q[key], q["fp64"], 0.5)
        rows.append(row)
    out["stopped"] = stopped
    for ctx in ctxs.values():
        ctx.close()
    out["vortex_gpu"] = {"case": big.name, "points": big.npts, "rows": rows}
    small = cases.vortex(nx=96, ny=64, nz=32)
    o = po.Oracle(small, threads=os.cpu_count() or 1)
    gs = {"fp64": api.Context(small), "fast": api.Context(small, precision=api.FP64_FAST),
          "fp32": api.Context(small, precision=api.FP32_MIXED)}
    res, done = [], 0
    for n in (50, 200, 1000):
        o.step(n - done)
        qo = o.state(0)
        row = {"steps": n}
        for key, g in gs.items():
            g.step(n - done)
            row[key] = state_errors(g.state(0), qo, 0.5)
        done = n
        res.append(row)
    for g in gs.values():
        g.close()
    out["vortex_vs_oracle"] = {"case": small.name, "points": small.npts, "rows": res,
                               "oracle_finite_at_1000": bool(np.isfinite(o.state(0)).all())}
    out["note"] = ("per conserved variable (rho, rho u, rho v, rho w, rho E); momentum components against "
                   "||rho|| * 0.5 where that exceeds their own norm (rho w is zero by symmetry)")
    return out


def smi_device(local):
    """The device that nvidia-smi and NVML should read for CUDA device `local`:
    its PCI bus id (domain:bus:device.function, as torch reports it), which
    names the same GPU whatever CUDA_VISIBLE_DEVICES maps, once a one-shot
    nvidia-smi query accepts it; else the index `local` as a string."""
    try:
        import torch
        pr = torch.cuda.get_device_properties(local)
        bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
        r = subprocess.run(["nvidia-smi", "-i", bus, "--query-gpu=index", "--format=csv,noheader"],
                           capture_output=True, text=True, timeout=10)
        if r.returncode == 0 and r.stdout.strip():
            return bus
    except Exception:
        pass
    return str(local)


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", gpu, f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def wait_first(self, timeout=2.0):
        """Returns once nvidia-smi has written its first sample (it starts slowly),
        so that a timed region of a few milliseconds still gets a record."""
        t0 = time.time()
        while self.p is not None and time.time() - t0 < timeout:
            if os.path.getsize(self.f.name) > 0:
                return
            time.sleep(0.02)

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except Exception:
                continue
            for i, nm in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 200 ms"}


class NvmlClocks:
    """SM clock and clock event reasons read through NVML (read-only queries)
    every `period` seconds on a thread between start() and stop(), so that a
    timed region shorter than nvidia-smi's sampling interval still gets samples
    taken under its load. Any NVML failure leaves it without samples, and
    summary() returns None."""

    # NVML clock event reason bits
    MASKS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, gpu, index=0, period=0.01, nvml=None):
        """gpu: a PCI bus id or an index, as smi_device gives it; index: the
        NVML index read when gpu is not a bus id NVML accepts."""
        self.rows, self.period, self.thread = [], period, None
        self.stop_ev = threading.Event()
        self.nv = None
        try:
            if nvml is None:
                import pynvml as nvml
            nvml.nvmlInit()
            try:
                self.h = nvml.nvmlDeviceGetHandleByPciBusId(str(gpu)) if ":" in str(gpu) else None
            except Exception:
                self.h = None
            if self.h is None:
                self.h = nvml.nvmlDeviceGetHandleByIndex(int(index))
            self.mx = float(nvml.nvmlDeviceGetMaxClockInfo(self.h, nvml.NVML_CLOCK_SM))
            self.reasons = getattr(nvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nvml.nvmlDeviceGetCurrentClocksThrottleReasons
            self.nv = nvml
        except Exception:
            self.nv = None

    def _poll(self):
        nv = self.nv
        while not self.stop_ev.is_set():
            try:
                self.rows.append((float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)),
                                  int(self.reasons(self.h))))
            except Exception:
                return
            self.stop_ev.wait(self.period)

    def start(self):
        if self.nv is not None:
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()

    def stop(self):
        if self.thread is not None:
            self.stop_ev.set()
            self.thread.join(timeout=2.0)
        if self.nv is not None:
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.rows:
            return None
        reasons = sorted(k for k, m in self.MASKS.items() if any(r & m for _, r in self.rows))
        return {"sm_mhz": float(np.median([s for s, _ in self.rows])), "sm_max_mhz": self.mx,
                "reasons": reasons, "samples": len(self.rows),
                "source": f"NVML, every {self.period * 1e3:.0f} ms during the timed steps"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))

    if args.mode == "cpu":
        if rank == 0:
            print(json.dumps(cpu_mode(args)), flush=True)
        return 0

    if args.impl == "reference":
        if rank != 0:
            return 0
        from canard_b200 import cases
        threads = os.cpu_count() or 1
        case_list, all_cases, workload = workload_cases(args, cases)
        v, secs = oracle_rate(case_list, args.steps, args.warmup, threads)
        npts = sum(c.npts for c in case_list)
        sample = (f"the whole workload ({len(case_list)} case(s), {npts} points): {args.warmup} warm-up and "
                  f"{args.steps} timed full reference time steps, FP64, OpenMP over lines on the host CPU")
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mpoint-steps/s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs * 1e3 / args.steps,
                "higher_is_better": True, "scaling": "weak" if args.config != "batched" else "strong",
                "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded analytic initial conditions; curv4 adds seeded velocity noise)",
                "config": config_dict(args, workload, len(case_list), npts, npts, 1),
                "cpu_baseline": {"value": v, "unit": "Mpoint-steps/s", "cores": threads,
                                 "kind": "port", "sample": sample},
                "e2e": {"value": v, "unit": "Mpoint-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from canard_b200 import api, cases

    if args.mode == "kernels":
        print(json.dumps(kernels_mode(args, api, cases, torch)), flush=True)
        return 0
    if args.mode == "accuracy":
        print(json.dumps(accuracy_mode(args, api, cases, torch)), flush=True)
        return 0
    if args.warmup < 3:
        raise SystemExit("at least 3 warm-up steps")
    case_list, all_cases, workload = workload_cases(args, cases, world, rank)
    prec = {"fp32": api.FP32_MIXED, "fast": api.FP64_FAST}.get(args.precision, api.FP64)
    ctx = api.Context(case_list, precision=prec)
    tuning = tune_context(ctx, args)
    # a non-default stream: the library launches on it and the CUDA events
    # below are recorded on it (handle 0 would mean the context's own stream)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    npts = sum(c.npts for c in case_list)
    if args.config == "batched":
        job_points, scaling = sum(c.npts for c in all_cases), "strong"
    else:
        job_points, scaling = world * npts, "weak"

    def barrier():
        if dist is not None:
            dist.barrier()

    ctx.step(args.warmup)
    dev = smi_device(local) if rank == 0 else None
    clk = Clocks(dev) if rank == 0 else None
    if clk:
        clk.wait_first()
    nclk = NvmlClocks(dev, local) if rank == 0 else None
    barrier()
    torch.cuda.synchronize()
    n0 = ctx.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if nclk:
        nclk.start()
    e0.record(stream)
    ctx.step(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    if nclk:
        nclk.stop()
    barrier()
    clocks = clk.stop() if clk else None
    # NVML's samples fall inside the timed steps; nvidia-smi's 200 ms record is
    # kept when NVML gave none
    in_region = nclk.summary() if nclk else None
    if in_region is not None:
        if clocks is not None:
            in_region["nvidia_smi"] = clocks
        clocks = in_region
    ms = e0.elapsed_time(e1)
    launches = ctx.launch_count() - n0
    if dist is not None:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = job_points * args.steps / (ms / 1e3) / 1e6

    # per-family device time (the reference's timers as CUDA events), one step
    ctx.set_timers(True)
    ctx.step(1)
    fam = ctx.timers()
    ctx.set_timers(False)
    tot = sum(f["ms"] for f in fam.values())
    peak, peak_kind = peaks()
    # DRAM bytes per algorithmic byte of each family's kernel from an ncu
    # capture of a smaller case (FP64 kernels), scaled to this launch
    ratios = {}
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath) and args.precision != "fp32":
        try:
            ratios = {k: v["dram_bytes_per_algorithmic_byte"] for k, v in json.load(open(tpath)).items()}
        except Exception:
            ratios = {}

    def family_roofline(name, kernel):
        f = fam[name]
        per = f["bytes"] / f["launches"]
        achieved = per / (f["ms"] / f["launches"] / 1e3) / 1e9
        return {"bound": "hbm", "kernel": f"{kernel} ({name})", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": ratios[name] * per if name in ratios else None,
                "algorithmic_bytes_per_launch": per, "share_of_step": f["ms"] / tot if tot else 0.0}

    # the dominant kernel: the single kernel with the largest share of the step
    # (each family is one kernel; the line solves are one kernel per direction)
    kernel_of = {"flux_components": "k_flux_visc_pairs" if args.precision == "fp32" else "k_flux_visc",
                 "rk_update": "k_rk_next", "primitives": "k_prim"}
    cands = [(k, v) for k, v in fam.items() if v["launches"] and v["bytes"] > 0
             and (k in kernel_of or k.startswith(("deriv", "filter")))]
    dom_name = max(cands, key=lambda kv: kv[1]["ms"])[0]
    def line_kernel(name):
        """The line kernels of a family: the autotuner's kinds for its groups."""
        op, d = name.split("_")
        groups = ("filter",) if op == "filter" else ("viscous", "flux")
        kinds = sorted({t["kind"] for t in (tuning or []) if t["dir"] == d and t["group"] in groups})
        return "line solve, " + ("/".join(kinds) if kinds else "default kinds")

    roofline = family_roofline(dom_name, kernel_of.get(dom_name) or line_kernel(dom_name))
    line_fams = {k: v for k, v in fam.items() if k.startswith(("deriv", "filter")) and v["launches"]}
    ln = max(line_fams, key=lambda k: line_fams[k]["ms"])
    roofline_line = family_roofline(ln, line_kernel(ln))
    lb = sum(v["bytes"] for v in line_fams.values())
    lms = sum(v["ms"] for v in line_fams.values())
    roofline_line["all_line_solves_gbs"] = lb / (lms / 1e3) / 1e9
    roofline_line["all_line_solves_share"] = lms / tot if tot else 0.0

    # end to end through the C ABI: pinned host state in and out every step
    hosts = []
    for ci, c in enumerate(case_list):
        for bi, b in enumerate(c.blocks):
            qh = torch.empty((5,) + b.shape, dtype=torch.float64, pin_memory=True)
            qh.copy_(torch.from_numpy(ctx.state(bi, ci)))
            hosts.append((ci, bi, qh, qh.numpy()))
    # one untimed step through the same call: its first use sets up the
    # staging buffer and copy streams
    ctx.step_host(1, [h[3] for h in hosts], [(h[0], h[1]) for h in hosts])
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    # every step: the state in from pinned host memory, the step, its result
    # back out (canard_step_host pipelines the two directions in chunks)
    ctx.step_host(args.e2e_steps, [h[3] for h in hosts], [(h[0], h[1]) for h in hosts])
    f1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ems = max(f0.elapsed_time(f1), wall * 1e3)
    if dist is not None:
        t = torch.tensor([ems], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ems = float(t.item())
    e2e = {"value": job_points * args.e2e_steps / (ems / 1e3) / 1e6, "unit": "Mpoint-steps/s",
           "h2d_bytes_per_step": int(sum(h[2].numel() for h in hosts) * 8),
           "d2h_bytes_per_step": int(sum(h[2].numel() for h in hosts) * 8),
           "steps": args.e2e_steps}

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras and args.config == "tgv" and args.precision != "fp32":
        ctx.close()
        torch.cuda.empty_cache()
        if args.precision == "fast":
            extras["fp64_bit_exact"] = precision_extra(args, api, cases, torch, stream, api.FP64)
            v64 = extras["fp64_bit_exact"]["value"]
        else:
            v64 = value
        f32 = precision_extra(args, api, cases, torch, stream, api.FP32_MIXED)
        f32["speedup_vs_fp64_bit_exact"] = f32["value"] / v64
        if args.precision == "fast":
            f32["speedup_vs_fp64_fast"] = f32["value"] / value
        extras["fp32_mixed"] = f32
        extras["batched"] = batched_extra(args, api, cases, torch, stream)
        torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        ctx.close()
        torch.cuda.empty_cache()
        th = os.cpu_count() or 1
        v, _ = oracle_rate(case_list, args.cpu_steps, 1, th)
        sample = (f"the timed workload itself ({npts} points): 1 warm-up and {args.cpu_steps} timed full reference "
                  "time steps, FP64, OpenMP over lines")
        cpu = {"value": v, "unit": "Mpoint-steps/s", "cores": th, "kind": "port", "sample": sample}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "Mpoint-steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": scaling, "vs_baseline": None, "dtype": "f32+f64" if args.precision == "fp32" else "f64",
                "data": "synthetic (seeded analytic initial conditions; curv4 adds seeded velocity noise)",
                "config": config_dict(args, workload, len(case_list), job_points, npts, world),
                "autotuned": not args.no_autotune,
                "roofline": roofline, "roofline_line_solve": roofline_line,
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clocks,
                "families": {k: {"ms_per_step": v["ms"], "share": v["ms"] / tot if tot else 0.0,
                                 "launches": v["launches"]} for k, v in fam.items() if v["launches"]}}
        if tuning is not None:
            line["autotune"] = tuning
        line.update(extras)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
