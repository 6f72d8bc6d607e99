"""Regenerates explosion_masks_81sq_N5.npz: the troubled-cell mask of the
2D N=5 Euler explosion on 81 x 81 outflow cells (DMP delta0 1e-4, eps 1e-3,
one helper layer, no cure steps, explosion centre from seed 0) after every
time step to t = 0.2, computed by the reference's own generic kernels
(oracle/_ref, parity build, driven by the oracle's limiting harness) and by
the oracle's plain-C restatement of the same kernels, both on all host
threads.

  python tests/golden/make_explosion_masks.py [--threads N]

About ten minutes of CPU time. The output is committed; the GPU test
tests/test_gpu_limiter_full.py replays the same run on the device and
compares the mask after every step with these.

Writes (step k = 1 .. steps; index 0 holds the initial statuses):
  status    uint8 [steps+1, 6561]  limiter status of every cell (0 DG, 1 and
                                   2 helper layers, 3 troubled), reference
  t, dt     float64 [steps+1]      time stamp and step size after each step
  irregular int64 [steps+1]        irregular steps so far
  sweeps    int64 [steps+1]        Picard sweeps so far
  status_oracle, sweeps_oracle     the same from the plain-C restatement: the
                                   two sequential CPU codes differ only in the
                                   order of floating-point operations, which
                                   shows where the run is sensitive to it
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))

CELLS = (81, 81)
ORDER = 5
T_END = 0.2
SEED = 0
OUT = os.path.join(HERE, "explosion_masks_81sq_N5.npz")


def run(impl, threads):
    import pyoracle
    from exahype_b200 import problems
    luh, fv, _ = problems.explosion(2, ORDER, CELLS, seed=SEED)
    cls = pyoracle.RefLimitingMesh if impl == "ref" else pyoracle.LimitingMesh
    o = cls(2, ORDER, CELLS, [1.0, 1.0], 0, helper_layers=1, cure_steps=0, nthreads=threads)
    o.set_solution(luh)
    o.set_fv_initial(fv)
    o.init(0.0)
    status, t, dt, irr, sw = [], [], [], [], []

    def record():
        st = o.state()
        status.append(o.status().astype(np.uint8))
        t.append(st["t"])
        dt.append(st["dt"])
        irr.append(st["irregular_steps"])
        sw.append(st["picard_sweeps"])
        return st

    st = record()
    t0 = time.time()
    # the reference's loop: step while t < t_end and dt > 0 (no clamp)
    while st["t"] < T_END and st["dt"] > 0:
        o.step(1)
        st = record()
        if len(t) % 100 == 0:
            print("step %d t %.5f (%.0f s)" % (len(t) - 1, st["t"], time.time() - t0), flush=True)
    return dict(status=np.array(status), t=np.array(t), dt=np.array(dt), irregular=np.array(irr, dtype=np.int64),
                sweeps=np.array(sw, dtype=np.int64))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=OUT)
    a = ap.parse_args()
    r = run("ref", a.threads)
    o = run("oracle", a.threads)
    assert len(o["t"]) == len(r["t"]), "the two CPU runs take different numbers of steps"
    r["status_oracle"], r["sweeps_oracle"] = o["status"], o["sweeps"]
    np.savez_compressed(a.out, **r)
    print("%s: %d steps to t = %.6f, %d irregular, %d sweeps, %d bytes" % (
        a.out, len(r["t"]) - 1, r["t"][-1], r["irregular"][-1], r["sweeps"][-1], os.path.getsize(a.out)))
