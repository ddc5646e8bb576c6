"""Counts the work of one complete 30-day run of the 3D benchmark with the
FP64 CPU oracle (test infrastructure; no product library is loaded) and
writes oracle/richards3d_30day_work.json.

The CPU baseline of bench.py times the oracle's unit costs on the 3D mesh
(a residual, a preconditioner set-up, a GMRES cycle) in a bounded sample and
scales them by these counts to the whole run, because the whole run takes
15 minutes of 8 host cores.  The oracle is deterministic (fixed summation
orders, static OpenMP schedules), so the counts do not depend on the host or
the thread count; the wall time recorded beside them validates the cost
model on the host that made the file.

usage: python oracle/work_counts.py [days]
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from oracle.pyoracle import Oracle, make_problem, opts  # noqa: E402


def main(days=30.0):
    p = make_problem("richards3d")
    o = Oracle(p)
    y0 = o.initial_head()
    op = opts(krylov_dim=40, max_order=5)
    t0 = time.perf_counter()
    rc, _, st = o.integrate(op, 148, 0.0, days * 86400.0, y0)
    wall = time.perf_counter() - t0
    if rc != 0:
        raise SystemExit(f"oracle run failed: {rc} {st}")
    tm, cnt = o.timers()
    tr = o.trace()
    # orthogonalisation work: iteration j of a cycle costs j + 1 dot/axpy
    # pairs, so a solve of n iterations (cycles of at most 40) costs
    # sum (j + 1); a step's Krylov iterations are split evenly over its
    # Newton solves
    s2 = 0.0
    for nli, nni in zip(tr["nli"], tr["nni"]):
        nni = max(int(nni), 1)
        per = nli / nni
        full, rest = divmod(per, 40)
        s2 += nni * (full * 40 * 41 / 2 + rest * (rest + 1) / 2)
    out = {
        "workload": f"richards3d 100x100x20 hex -> 6 tets (214,221 nodes), {days:g} days, rtol = atol = 1e-6, "
                    "GMRES(40), 148 ILU blocks, FP64 CPU oracle",
        "simulated_s": days * 86400.0,
        "counts": cnt,
        "stats": {k: st[k] for k in ("nst", "nni", "nli", "npe", "nps", "nre", "ncfn", "netf")},
        "orth_pairs": s2,
        "measured": {"wall_s": wall, "threads": Oracle.threads(), "time_split_s": tm},
    }
    path = os.path.join(HERE, f"richards3d_{days:g}day_work.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main(float(sys.argv[1]) if len(sys.argv) > 1 else 30.0)
