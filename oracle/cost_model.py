"""CPU baseline of the 3D benchmark: the FP64 oracle's unit costs, measured
on the 214,221-node mesh in a bounded sample, times the work of one whole
30-day run as the oracle itself counts it (oracle/richards3d_30day_work.json,
made by oracle/work_counts.py).

TEST INFRASTRUCTURE: used only by bench.py's CPU legs (the timed CPU
baseline and the reference arm); it loads the oracle's library, never the
product library.

One sample, at the hydrostatic initial state of the run, with the run's
options (148 ILU blocks, GMRES(40)):
  * a Newton residual evaluation;
  * a preconditioner set-up (30 coloured residuals + block ILU(0) factor);
  * one GMRES cycle of 40 iterations (tolerance 0), which gives the cost of a
    J*v product, a preconditioner apply, and the orthogonalisation per
    (j + 1) dot/axpy pairs of iteration j.
The run's time is then
  newton_residuals * t_res + jv * t_jv + setups * t_setup + applies * t_apply
  + orth_pairs * t_pair,
with the counts of the file.  The controller's own O(N) vector work (about
half a per cent of the oracle's run) is left out.
"""
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
WORK_FILE = os.path.join(HERE, "richards3d_30day_work.json")


def work():
    with open(WORK_FILE) as f:
        return json.load(f)


class Sampler:
    """the 3D problem and its oracle, built once (about 10 s)"""

    def __init__(self):
        from oracle.pyoracle import Oracle, make_problem

        self.problem = make_problem("richards3d")
        self.oracle = Oracle(self.problem)
        self.y0 = self.oracle.initial_head()
        self.work = work()

    def sample(self):
        """one bounded sample; returns (modelled seconds of the whole run,
        unit costs, wall seconds the sample took)"""
        o, y = self.oracle, self.y0
        w0 = time.perf_counter()
        yp = np.zeros_like(y)
        ewt = 1.0 / (1e-6 * np.abs(y) + 1e-6)
        o.begin_step(0.0, y, yp)
        t = time.perf_counter()
        F0 = o.residual(0.0, y, yp)
        t_res = time.perf_counter() - t
        cj, h = 1.0 / 100.0, 100.0
        t = time.perf_counter()
        o.psetup(0.0, cj, h, y, yp, F0, ewt, 148)
        t_setup = time.perf_counter() - t
        o.timers(reset=True)
        o.gmres(cj, y, yp, F0, ewt, F0, m=40, max_restarts=0, tol=0.0)
        tm, cnt = o.timers(reset=True)
        its = max(cnt["krylov_iterations"], 1)
        unit = {
            "newton_residual_s": t_res,
            "setup_s": t_setup,
            "jv_s": tm["jv"] / max(cnt["jv"], 1),
            "apply_s": tm["ilu_apply"] / max(cnt["applies"], 1),
            "orth_pair_s": tm["krylov_other"] / (its * (its + 1) / 2),
        }
        c = self.work["counts"]
        total = (c["newton_residuals"] * unit["newton_residual_s"] + c["jv"] * unit["jv_s"]
                 + c["setups"] * unit["setup_s"] + c["applies"] * unit["apply_s"]
                 + self.work["orth_pairs"] * unit["orth_pair_s"])
        return total, unit, time.perf_counter() - w0
