#!/usr/bin/env python
"""Benchmark: simulated seconds per wall second of the 200k-node 3D Richards
case (101 x 101 x 21 nodes, 1.2 M tetrahedra, lognormal Ks, 30 days,
Newton tolerance from rtol = atol = 1e-6) on B200.

One step = one complete 30-day integration from the hydrostatic initial
state (variable-order BDF, Newton-GMRES(40), block-ILU(0)).  The headline
``value`` is the learned + mixed-precision path: the per-node MLP proposes
the Newton initial iterate (kept only when its FP64 residual beats the BDF
predictor's); the block-ILU(0) factor and apply, the Krylov basis and the
Krylov operator -- the preconditioner set-up's assembled difference-quotient
Jacobian, applied in one fused persistent launch per GMRES cycle -- run in
FP32; the residual, Newton update, least squares and stopping tests stay
FP64.  The state is resident in HBM.  The MLP is trained before the timed
region on a plain FP64 trajectory of a different Ks realisation.  The plain
FP64 path (the reference's Jacobian-free method: J v as the difference
quotient of the FP64 residual), the FP32 Jacobian-free path and the FP32
assembled path without the learned iterate are timed the same way and
reported beside it.  ``e2e`` is the same metric through
fvm_integrate_host (host buffers, H2D of y0 and D2H of the final head inside
the timed region).

Multi-GPU (torchrun): every rank integrates its own replica (a different Ks
seed) with no data-path collective -- the problem does not shard -- so the
value is replicas x simulated seconds / max-over-ranks time ("weak").

``--impl reference`` times the FP64 CPU oracle (the reference path restated
in C++, OpenMP on all host cores) on the same 30-day workload: each step
measures the oracle's unit costs on the 3D mesh in a bounded sample and
scales them by the oracle's own counted work of the whole run
(oracle/cost_model.py); the reference itself cannot be built (no
SUNDIALS/MKL/minlin/MPI).  That process loads only the oracle's library.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "sim-s/wall-s, 200k-node 3D Richards @1e-6: learned+FP32 vs plain FP64, 1×B200"
WORKLOAD = "richards3d 101x101x21 nodes / 1.2M tets (214,221 nodes), one 30-day run per step"
# the workload both arms time: the same dict in the line of each
CONFIG = {"workload": WORKLOAD, "rtol": 1e-6, "atol": 1e-6, "simulated_s_per_step": 30 * 86400.0,
          "l2": "inputs larger than L2 (331 MB per residual evaluation)"}
# DRAM bytes (read + write) of one residual evaluation of this workload --
# node pass 8.3 MB, element pass 62.6 MB, gather 13.1 MB -- as measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum) on the --profile-case
# residual workload.  The algorithmic 331.7 MB assume stored face
# coefficients; the rebuilt-geometry element pass reads a fifth of that.
CHAIN_DRAM_BYTES = 84.0e6
# DRAM bytes (read + write) of one k_arnoldi_fused launch, as measured by ncu
# on the --profile-case fused workload: launches 101 (2-3 Arnoldi steps,
# 44.4 MB read, 0.4 MB written) and 102 (a full 40-step cycle, 44.4 MB read,
# 2.3 MB written) of the 10-day run, whose mean length (21 steps) is the
# 30-day run's mean; their mean is used.  The operator and the FP32 basis stay
# in L2 between steps, so this stays far below the algorithmic bytes, which
# count every L2 -> SM pass.
FUSED_DRAM_BYTES = 45.7e6
UNIT = "sim-s/wall-s"


def peaks():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region"""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.lines = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
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
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def max_over_ranks(x, ws, dev):
    from fvmpor_b200.replicas import max_over_ranks as mor

    return x if ws == 1 else mor(x, dev)


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def cpu_baseline_sample(samples=2):
    """the FP64 CPU oracle's time for the whole 30-day run, from its unit
    costs on the 3D mesh (bounded samples) times its own counted work of the
    run (oracle/cost_model.py); returns (sim-s/wall-s, modelled seconds,
    unit costs, sample wall seconds, threads)"""
    from oracle.cost_model import Sampler
    from oracle.pyoracle import Oracle

    sm = Sampler()
    sm.sample()   # the first set-up also builds the pattern and colouring
    runs = [sm.sample() for _ in range(samples)]
    total = float(np.median([r[0] for r in runs]))
    unit = runs[-1][1]
    return sm.work["simulated_s"] / total, total, unit, sum(r[2] for r in runs) / len(runs), Oracle.threads()


def error_vs_oracle(fb, torch, ph, y0, trace, n_steps, precision_paths, newton_tol=1e-5):
    """Replay the first n_steps accepted steps of a GPU run (step sizes and
    orders fixed, every corrector solved to ||delta||_wrms <= newton_tol) on
    the GPU, once per path in precision_paths, and in the FP64 CPU oracle's
    independent replay; returns the largest relative head difference of each
    path against the oracle"""
    from oracle.pyoracle import Oracle

    steps = trace[:n_steps]
    h0 = float(steps["h"][0])
    nb = fb.Preconditioner(ph).info()["nblocks"]
    orc = Oracle(ph.problem)
    y0h = y0.cpu().numpy()
    t = time.perf_counter()
    rc, yr, st = orc.replay(fb.default_opts(krylov_dim=40, max_order=5), nb, 0.0, y0h, h0, steps,
                            newton_tol=newton_tol)
    oracle_s = time.perf_counter() - t
    out = {"steps": int(n_steps), "t_end_s": float(st["t"]), "newton_tol_wrms": newton_tol, "oracle_rc": rc,
           "oracle_s": oracle_s}
    for name, kw in precision_paths.items():
        yg = torch.empty_like(y0)
        rcg, stg = fb.Integrator(ph, krylov_dim=40, max_restarts=5, max_order=5, **kw).replay(
            0.0, y0, h0, steps, yg, newton_tol=newton_tol)
        out[name] = float(np.abs(yg.cpu().numpy() - yr).max() / np.abs(yr).max())
        out[name + "_rc"] = rcg
    del orc
    return out


def train_predictor(fb, torch, dev, seed, horizon):
    """Learned Newton iterate: record a plain FP64 trajectory of another Ks
    realisation (same mesh shape and soil), then fit the per-node MLP to its
    scaled Newton corrections with the device's own forward/backward/Adam
    kernels.  Runs before (outside) the timed region; returns the parameter
    vector and a summary."""
    t0 = time.perf_counter()
    pt = fb.make_problem("richards3d", seed=seed)
    pht = fb.Physics(pt)
    y0 = torch.empty(pt.n_nodes, dtype=torch.float64, device=dev)
    pht.initial_head(y0)
    ye = torch.empty_like(y0)
    cap = 6_000_000
    X = torch.zeros((cap, 8), dtype=torch.float32, device=dev)
    Y = torch.zeros(cap, dtype=torch.float32, device=dev)
    rec = fb.Integrator(pht, krylov_dim=40, max_restarts=5, precision=0, max_order=5)
    rc, st, cnt = rec.integrate_record(0.0, horizon, y0, ye, X, Y, stride=29)
    if rc != 0 or cnt < 1000:
        raise RuntimeError(f"training trajectory failed rc={rc} samples={cnt}")
    t_rec = time.perf_counter() - t0
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    perm = torch.randperm(cnt, device=dev, generator=gen)
    Xs, Ys = X[:cnt][perm].contiguous(), Y[:cnt][perm].contiguous()
    del X, Y
    pr = fb.Predictor(pht)
    pr.init(Xs, seed=seed)
    t1 = time.perf_counter()
    rc, hist = pr.train(Xs, Ys, epochs=6, batch=8192, lr=2e-3)
    torch.cuda.synchronize()
    t_fit = time.perf_counter() - t1
    if rc != 0:
        raise RuntimeError(f"predictor training failed rc={rc}")
    P = pr.get_params()
    info = {"train_seed": seed, "samples": int(cnt), "epochs": 6, "loss_first_epoch": float(hist[0]),
            "loss_last_epoch": float(hist[-1]), "record_s": t_rec, "fit_s": t_fit,
            "trajectory_steps": st["nst"]}
    pht.close()
    del Xs, Ys
    torch.cuda.empty_cache()
    return P, info


def profile_case(name, days=10.0):
    """Small fixed workloads of single kernels for profiler captures (not a
    bench line): 'residual' evaluates the residual five times at the
    hydrostatic head; 'precond' sets up the FP32 preconditioner three times
    and applies it 20 times after each set-up; 'krylov' integrates the first
    10 days with the FP32 Krylov path (about 120 steps, 16 Krylov iterations
    per Newton solve by the end); 'fused' integrates the first --days days
    with the FP32 assembled Krylov operator (one fused launch per GMRES
    cycle)."""
    import torch

    import fvmpor_b200 as fb

    dev = torch.device("cuda", 0)
    p = fb.make_problem("richards3d")
    ph = fb.Physics(p)
    N = p.n_nodes
    y = torch.empty(N, dtype=torch.float64, device=dev)
    ph.initial_head(y)
    yp = torch.zeros_like(y)
    r = torch.empty_like(y)
    if name == "residual":
        for _ in range(5):
            ph.residual(0.0, y, yp, r)
    elif name == "precond":
        ph.begin_step(0.0, y, yp)
        ph.residual(0.0, y, yp, r)
        pc = fb.Preconditioner(ph)
        ewt = torch.full_like(y, 1e6)
        v = torch.randn(N, dtype=torch.float64, device=dev, generator=torch.Generator(device=dev).manual_seed(1))
        z = torch.empty_like(y)
        for _ in range(3):
            pc.setup(0.0, 1e-2, 100.0, y, yp, r, ewt, precision=1)
            for _ in range(20):
                pc.apply(v, z)
    elif name == "krylov":
        ye = torch.empty_like(y)
        fb.Integrator(ph, krylov_dim=40, max_restarts=5, precision=1, max_order=5).integrate(0.0, 10 * 86400.0, y, ye)
    else:
        ye = torch.empty_like(y)
        fb.Integrator(ph, krylov_dim=40, max_restarts=5, precision=1, krylov_operator=1, max_order=5).integrate(
            0.0, days * 86400.0, y, ye)
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": name, "ok": True}))


def run_reference(args):
    """FP64 CPU oracle (the reference path restated in C++, OpenMP on every
    host core; the reference itself needs SUNDIALS, MKL, minlin and MPI and
    does not build) on the same workload: one step is one bounded sample of
    the oracle's unit costs on the 214,221-node mesh, scaled to the whole
    30-day run by the oracle's own counted work.  Only the oracle's library is
    loaded in this process."""
    import numpy as np  # noqa: F401  (used by the sampler)

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.cost_model import Sampler
    from oracle.pyoracle import Oracle

    sm = Sampler()
    for _ in range(args.warmup):
        sm.sample()
    totals, walls = [], []
    for _ in range(args.steps):
        tot, unit, wall = sm.sample()
        totals.append(tot)
        walls.append(wall)
    total = float(statistics.median(totals))
    value = sm.work["simulated_s"] / total
    threads = Oracle.threads()
    meas = sm.work["measured"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(walls) / len(walls),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded 3D jittered Kuhn mesh, lognormal Ks)",
        "config": dict(CONFIG),
        "cpu_baseline": {
            "value": value, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": ("unit costs of the FP64 oracle on the 214,221-node mesh (Newton residual, preconditioner "
                       "set-up, J*v, apply, orthogonalisation from one 40-iteration GMRES cycle) per step, times the "
                       "oracle's own counted work of the whole 30-day run "
                       f"({sm.work['counts']['steps']} steps, {sm.work['counts']['krylov_iterations']} Krylov "
                       "iterations, oracle/richards3d_30day_work.json); the model was checked against a measured "
                       f"whole run ({meas['wall_s']:.0f} s on {meas['threads']} threads of the host that made the file, "
                       "where samples of the model gave 470-510 s)"),
            "modelled_run_s": total, "unit_costs_s": unit,
        },
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# the other benchmark configurations (not the headline line): generator
# name, horizon, Krylov dimension, simulated-time multiplier (ensemble
# members), and the paths timed (the first is the line's value)
WORKLOADS = {
    "plane": dict(problem="richards2d", days=1.0, m=30, desc="richards2d 81x41 jittered Delaunay (3,321 nodes), "
                  "2 layers, ponded strip, 1 day, GMRES(30), rtol = atol = 1e-6",
                  paths={"plain_fp64": dict(precision=0), "plain_fp64_graph": dict(precision=0, graph=1),
                         "fp32_jacobian_free": dict(precision=1),
                         "fp32_jacobian_free_graph": dict(precision=1, graph=1),
                         "fp32_assembled": dict(precision=1, krylov_operator=1)}),
    "ensemble": dict(problem="ensemble2d", days=1.0, m=30, batch=True,
                     desc="ensemble2d: 256 independent 2D meshes of 2k-40k nodes (5.37 M nodes), own lognormal Ks, "
                          "1 day, FP64 residual + FP32 preconditioner, every member with its own step sequence",
                     paths={"fp32_assembled": dict(precision=1, krylov_operator=1),
                            "fp32_jacobian_free_graph": dict(precision=1, graph=1),
                            "fp32_jacobian_free": dict(precision=1)}),
    "box1m": dict(problem="richards3d_1m", days=30.0, m=40, desc="richards3d_1m: 200x200x25 hex -> 6 tets "
                  "(1,050,426 nodes), lognormal Ks, 30 days, GMRES(40)",
                  paths={"fp32_assembled": dict(precision=1, krylov_operator=1),
                         "fp32_jacobian_free": dict(precision=1), "plain_fp64": dict(precision=0)}),
}


def run_ensemble(args, wl):
    """the ensemble's members in their own contexts, integrated concurrently
    (fvm_integrate_batch, 16 host threads, one stream per member); the timed
    region is bracketed by events on the legacy default stream, which every
    member's (blocking) stream waits for and is waited on by; value = the
    simulated seconds all members reached per wall second"""
    import torch

    import fvmpor_b200 as fb

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    t = time.perf_counter()
    union = fb.make_problem(wl["problem"])
    members = [union.member(m) for m in range(len(union.member_ptr) - 1)]
    gen_s = time.perf_counter() - t
    # largest members first, so the threads finish together
    order = sorted(range(len(members)), key=lambda m: -members[m].n_nodes)
    t = time.perf_counter()
    phs = [fb.Physics(members[m]) for m in order]
    torch.cuda.synchronize()
    create_s = time.perf_counter() - t
    horizon = (args.days if args.days is not None else wl["days"]) * 86400.0
    y0 = []
    for ph in phs:
        v = torch.empty(ph.N, dtype=torch.float64, device=dev)
        ph.initial_head(v)
        y0.append(v)
    ye = [torch.empty_like(v) for v in y0]
    runs, stats = {k: [] for k in wl["paths"]}, {}
    for k, kw in wl["paths"].items():   # warm-up: every member's workspace
        fb.integrate_batch(phs, 0.0, horizon, y0, ye, n_threads=16, krylov_dim=wl["m"], max_restarts=5,
                           max_order=5, **kw)
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            for k, kw in wl["paths"].items():
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                rc, status, st = fb.integrate_batch(phs, 0.0, horizon, y0, ye, n_threads=16, krylov_dim=wl["m"],
                                                    max_restarts=5, max_order=5, **kw)
                e1.record()
                torch.cuda.synchronize()
                runs[k].append(e0.elapsed_time(e1))
                reached = sum(min(x["t"], horizon) for x in st)
                failed = [order[i] for i, r in enumerate(status) if r != 0]
                stats[k] = {"simulated_s": reached, "members_failed": len(failed), "failed_members": failed[:64],
                            "steps": sum(x["nst"] for x in st), "newton": sum(x["nni"] for x in st),
                            "krylov": sum(x["nli"] for x in st),
                            "failed_at_s": sorted(round(st[i]["t"], 1) for i, r in enumerate(status) if r != 0)[:64]}
    head = next(iter(wl["paths"]))
    cmp = {k: {"value": stats[k]["simulated_s"] / (float(np.median(v)) / 1e3), "ms_per_run": float(np.median(v)),
               "ms_each_run": v, "stats": stats[k]} for k, v in runs.items()}
    line = {"metric": f"sim-s/wall-s, {wl['desc']}, 1xB200", "value": cmp[head]["value"], "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": 1, "ms_per_step": cmp[head]["ms_per_run"], "higher_is_better": True,
            "dtype": "f64", "data": "synthetic (seeded meshes and Ks fields)",
            "config": {"workload": wl["desc"] if horizon == wl["days"] * 86400.0 else
                       wl["desc"] + f" (run to {horizon / 3600.0:g} h)", "members": len(members),
                       "nodes": union.n_nodes, "elements": union.n_elements, "simulated_s_per_member": horizon,
                       "host_threads": 16},
            "path": head, "paths": cmp, "preprocessing_s": {"generate": gen_s, "create_contexts": create_s},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    for ph in phs:
        ph.close()


def run_workload(args):
    """one of the other configurations at its stated size (1 GPU): every
    path of WORKLOADS[name] timed run by run, alternating, after one warm-up
    run each; value = the first path's simulated seconds (times the
    ensemble's members) per wall second of its median run"""
    import torch

    import fvmpor_b200 as fb

    wl = WORKLOADS[args.workload]
    if wl.get("batch"):
        run_ensemble(args, wl)
        return
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    t = time.perf_counter()
    prob = fb.make_problem(wl["problem"])
    gen_s = time.perf_counter() - t
    t = time.perf_counter()
    ph = fb.Physics(prob)
    torch.cuda.synchronize()
    create_s = time.perf_counter() - t
    members = len(prob.member_ptr) - 1 if prob.member_ptr is not None else 1
    horizon = (args.days if args.days is not None else wl["days"]) * 86400.0
    y0 = torch.empty(prob.n_nodes, dtype=torch.float64, device=dev)
    ph.initial_head(y0)
    ye = torch.empty_like(y0)
    integ = {k: fb.Integrator(ph, krylov_dim=wl["m"], max_restarts=5, max_order=5, **kw)
             for k, kw in wl["paths"].items()}
    for it in integ.values():
        rc, _ = it.integrate(0.0, horizon, y0, ye)
        if rc != 0:
            raise RuntimeError(f"warm-up run failed rc={rc}")
    runs = {k: [] for k in integ}
    stats = {}
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            for k, it in integ.items():
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                rc, st = it.integrate(0.0, horizon, y0, ye)
                e1.record()
                torch.cuda.synchronize()
                if rc != 0:
                    raise RuntimeError(f"{k} failed rc={rc} {st}")
                runs[k].append(e0.elapsed_time(e1))
                stats[k] = {q: st[q] for q in ("nst", "nni", "nli", "npe", "nre", "ncfn", "netf", "nsync")}
    head = next(iter(integ))
    cmp = {k: {"value": members * horizon / (float(np.median(v)) / 1e3), "ms_per_run": float(np.median(v)),
               "ms_each_run": v, "stats": stats[k],
               "host_waits_per_step": stats[k]["nsync"] / max(stats[k]["nst"], 1)} for k, v in runs.items()}
    y0h = y0.cpu().numpy()
    yh = np.zeros(prob.n_nodes)
    t = time.perf_counter()
    for _ in range(max(1, args.steps // 2)):
        integ[head].integrate_host(0.0, horizon, y0h, yh)
    e2e_s = (time.perf_counter() - t) / max(1, args.steps // 2)
    line = {"metric": f"sim-s/wall-s, {wl['desc']}, 1xB200", "value": cmp[head]["value"], "unit": UNIT,
            "n_gpus": 1, "steps": args.steps, "warmup": 1, "ms_per_step": cmp[head]["ms_per_run"],
            "higher_is_better": True, "dtype": "f64", "data": "synthetic (seeded meshes and Ks fields)",
            "config": {"workload": wl["desc"] if horizon == wl["days"] * 86400.0 else
                       wl["desc"] + f" (run to {horizon / 3600.0:g} h)", "members": members, "nodes": prob.n_nodes,
                       "elements": prob.n_elements, "simulated_s_per_member": horizon},
            "path": head, "paths": cmp,
            "preprocessing_s": {"generate": gen_s, "create_context": create_s},
            "preconditioner": fb.Preconditioner(ph).info(),
            "e2e": {"value": members * horizon / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 8 * prob.n_nodes,
                    "d2h_bytes_per_step": 8 * prob.n_nodes},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    ph.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--days", type=float, default=None,
                    help="simulated days per run (default: 30 for richards3d, the configuration's for the others)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--replay-steps", type=int, default=8,
                    help="steps of the headline run replayed against the CPU oracle for error_vs_oracle")
    ap.add_argument("--profile-case", choices=["residual", "precond", "krylov", "fused"],
                    help="run one small fixed workload for a profiler capture instead of the bench")
    ap.add_argument("--workload", default="richards3d", choices=["richards3d"] + sorted(WORKLOADS),
                    help="richards3d: the headline line; plane, ensemble, box1m: the other configurations at their "
                         "stated sizes (1 GPU)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload != "richards3d" and args.impl == "ours" and not args.profile_case:
        run_workload(args)
        return
    if args.days is None:
        args.days = 30.0
    if args.profile_case:
        profile_case(args.profile_case, args.days)
        return
    if args.impl == "reference":
        run_reference(args)
        return

    import torch

    import fvmpor_b200 as fb

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from fvmpor_b200.replicas import job_throughput, replica_seed

    prob = fb.make_problem("richards3d", seed=replica_seed(1, rank))
    horizon = args.days * 86400.0
    ph = fb.Physics(prob)
    N, T = prob.n_nodes, prob.n_elements
    y0 = torch.empty(N, dtype=torch.float64, device=dev)
    ph.initial_head(y0)
    yend = torch.empty_like(y0)
    P, train_info = train_predictor(fb, torch, dev, 1001 + rank, horizon)
    fb.Predictor(ph).set_params(P)
    common = dict(krylov_dim=40, max_restarts=5, max_order=5)
    # headline: learned iterate + FP32 factor, basis and assembled Krylov
    # operator (one fused launch per GMRES cycle)
    learned = fb.Integrator(ph, precision=1, krylov_operator=1, use_predictor=1, **common)
    assembled = fb.Integrator(ph, precision=1, krylov_operator=1, **common)
    fp32_dq = fb.Integrator(ph, precision=1, **common)
    plain = fb.Integrator(ph, precision=0, **common)

    def timed(integ, k, host=False, profile=False):
        y0h = y0.cpu().numpy()
        yh = np.zeros(N)
        barrier(ws)
        torch.cuda.synchronize()
        if profile:
            ph.profile(True)
        c0 = ph.counters()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stats = []
        e0.record()
        for _ in range(k):
            if host:
                rc, st = integ.integrate_host(0.0, horizon, y0h, yh)
            else:
                rc, st = integ.integrate(0.0, horizon, y0, yend)
            if rc != 0:
                raise RuntimeError(f"integration failed rc={rc} {st}")
            stats.append(st)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        c1 = ph.counters()
        prof = ph.profile_read() if profile else {}
        if profile:
            ph.profile(False)
        prof["_launches"] = (0.0, c1["launches"] - c0["launches"])
        barrier(ws)
        return max_over_ranks(ms, ws, dev), stats, prof

    for _ in range(args.warmup):
        learned.integrate(0.0, horizon, y0, yend)
    with ClockSampler(local) as clk:
        ms_learn, st_learn, cnt = timed(learned, args.steps)
    y_learn = yend.clone()
    trace_learn = learned.trace()
    # per-kernel CUDA-event profile on one more run outside the timed region
    # (the events themselves slow the run down)
    _, _, prof = timed(learned, 1, profile=True)
    st_prof = learned.trace()   # the trace belongs to the context: read it before the next run
    # the comparison paths are timed run by run, alternating, and reported as
    # the median run (each run is a whole 30-day integration; alternating
    # keeps a slow spell of the shared host from landing on one path only)
    k_extra = max(2, args.steps // 2)
    others = {"fp32_assembled_without_learned": assembled, "fp32_jacobian_free": fp32_dq, "plain_fp64": plain}
    for integ in others.values():
        integ.integrate(0.0, horizon, y0, yend)   # warm the FP32 and FP64 factor/basis buffers
    runs = {k: [] for k in others}
    st_o = {}
    with ClockSampler(local) as clk_cmp:
        for _ in range(k_extra):
            for name, integ in others.items():
                ms, st_o[name], _ = timed(integ, 1)
                runs[name].append(ms)
    y_plain = yend.clone()   # plain FP64 ran last
    ms_e2e, _, _ = timed(learned, k_extra, host=True)
    value = job_throughput(horizon * args.steps, ws, ms_learn / 1e3)
    e2e_value = job_throughput(horizon * k_extra, ws, ms_e2e / 1e3)
    head_diff = float((y_learn - y_plain).abs().max() / y_plain.abs().max())
    cmp = {}
    for name in others:
        med = float(np.median(runs[name]))
        cmp[name] = {"value": job_throughput(horizon, ws, med / 1e3), "ms_per_step": med, "runs": k_extra,
                     "ms_each_run": runs[name],
                     "stats": {k: st_o[name][0][k] for k in ("nst", "nni", "nli", "npe", "nre", "nsync")}}
    plain_value = cmp["plain_fp64"]["value"]
    cmp["plain_fp64"]["ratio_headline_over_plain"] = value / plain_value
    cmp["fp32_assembled_without_learned"]["clocks_comparison_runs"] = clk_cmp.summary()

    peak, peak_kind = peaks()
    # roofline of the dominant kernel, the fused Arnoldi cycle (delayed
    # reorthogonalisation): algorithmic bytes of Arnoldi step j (nv = j + 1
    # basis vectors) are the assembled operator (FP32 value + 4-byte column
    # per non-zero), per node the direction and the cj coefficient (4 B
    # each), ewt (8 B), two passes over the FP32 basis (8 nv B) and the new
    # basis vector and direction (8 B); the factor stays in shared memory
    # for the whole cycle.  Per launch = per cycle; the time is the kernel's
    # CUDA-event total over its launches of the profiled run.
    nnz = fb.Preconditioner(ph).info()["nnz"]
    nv_sum, n_ar = 0.0, 0
    for nli_s, nni_s in zip(st_prof["nli"], st_prof["nni"]):
        per = nli_s / max(int(nni_s), 1)   # Krylov iterations of each Newton solve of the step
        nv_sum += max(int(nni_s), 1) * per * (per + 1) / 2.0
        n_ar += int(nli_s)
    bytes_steps = n_ar * (8.0 * nnz + 24.0 * N) + 8.0 * N * nv_sum
    launches_k = max(int(prof["gram_schmidt"][1]), 1)
    fused_ms = prof["gram_schmidt"][0]
    achieved = bytes_steps / launches_k / (fused_ms / launches_k * 1e-3) / 1e9
    # residual evaluation chain (node pass + element pass + gather):
    # algorithmic bytes 36 B/node + 270 B/tet per evaluation
    alg_res = 36.0 * N + 270.0 * T
    n_eval = max(prof["element"][1], 1)
    chain_ms = (prof["node"][0] + prof["element"][0] + prof["gather"][0]) / n_eval
    achieved_res = alg_res / (chain_ms * 1e-3) / 1e9
    st0 = st_learn[0]
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_learn / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded 3D jittered Kuhn mesh, lognormal Ks by FFT)",
        "config": dict(CONFIG) if args.days == 30.0 else dict(CONFIG, workload=WORKLOAD.replace(
            "30-day", f"{args.days:g}-day"), simulated_s_per_step=horizon),
        "path": "learned Newton iterate (per-node MLP, BF16 weights / FP32 accumulation on tcgen05) + "
                "FP32 block-ILU(0), FP32 GMRES(40) basis and FP32 assembled Krylov operator (the "
                "set-up's difference-quotient Jacobian, one fused launch per GMRES cycle); FP64 "
                "residual, Newton update, least squares and tests",
        "parallelism": f"replicas x{ws}",
        "comparison_paths": cmp,
        "learned_predictor": dict(train_info, accepted_steps=st0["npred"]),
        "final_head_rel_diff_vs_plain_fp64": head_diff,
        "stats": {k: st0[k] for k in ("nst", "nni", "nli", "npe", "nps", "nre", "ncfn", "netf", "npred",
                                      "last_order", "nsync")},
        # host waits on the device per accepted step (the controller's
        # decisions still run on the host; every other launch is queued)
        "host_waits_per_step": st0["nsync"] / max(st0["nst"], 1),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": FUSED_DRAM_BYTES,
                     "kernel": "k_arnoldi_fused (one GMRES cycle: assembled operator, block-ILU(0) sweeps, "
                               "delayed-reorthogonalisation Gram-Schmidt, Givens)",
                     "algorithmic_bytes_per_launch": bytes_steps / launches_k,
                     "avg_ms": fused_ms / launches_k, "arnoldi_steps_per_launch": n_ar / launches_k,
                     "peak_kind": peak_kind},
        "roofline_residual": {"bound": "hbm", "achieved": achieved_res, "peak": peak, "unit": "GB/s",
                              "frac": achieved_res / peak, "traffic": CHAIN_DRAM_BYTES,
                              "kernel": "residual evaluation (node pass + element pass + node gather)",
                              "algorithmic_bytes_per_launch": alg_res, "avg_ms": chain_ms,
                              "peak_kind": peak_kind},
        "kernel_ms": {k: {"total_ms": v[0], "launches": v[1], "avg_us": 1e3 * v[0] / max(v[1], 1)}
                      for k, v in prof.items()},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * N, "d2h_bytes_per_step": 8 * N},
        "clocks": clocks,
        # the run is driven by one host thread: a busy host shows up as
        # slower, more variable runs
        "host_loadavg_1min": os.getloadavg()[0],
    }
    # every kernel launch of the library inside the timed region (counted by
    # the context: residual chain, Krylov, preconditioner, controller)
    line["gpu_launches"] = int(cnt["_launches"][1])
    line["kernel_ms"].pop("_launches", None)
    if rank == 0 and not args.no_cpu_baseline:
        # error of the final heads against the FP64 CPU oracle: the first
        # steps of the headline run replayed with tight correctors
        line["error_vs_oracle"] = error_vs_oracle(
            fb, torch, ph, y0, trace_learn, args.replay_steps,
            {"plain_fp64": dict(precision=0), "fp32_jacobian_free": dict(precision=1),
             "fp32_assembled": dict(precision=1, krylov_operator=1)})
        v, total, unit, wall, threads = cpu_baseline_sample()
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": "FP64 oracle unit costs on the 214,221-node mesh (2 bounded samples, "
                                          f"{wall:.1f} s each) times its counted work of the whole 30-day run "
                                          "(oracle/cost_model.py)",
                                "modelled_run_s": total}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ph.close()
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
