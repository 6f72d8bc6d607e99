"""The limiter benchmark workload run to its end on the GPU, with the
troubled-cell mask compared after every step against the reference's own
kernels.

Workload: 2D Euler N=5 circular explosion on 81 x 81 outflow cells, 11 x 11
MUSCL-Hancock subcells per cell, DMP delta0 1e-4 and epsilon 1e-3, one helper
layer, no cure steps, explosion centre from seed 0, run while t < 0.2 (the
reference's loop, no clamp of the last step).

Expected values: tests/golden/explosion_masks_81sq_N5.npz, the limiter
status of every cell after every step of the same run by the reference's
generic kernels compiled from its sources (oracle/_ref, parity build, driven
by the oracle's limiting harness), made by tests/golden/make_explosion_masks.py.

Bar: the status of every cell (troubled cells and both helper layers) equal
after every step; the same number of steps, irregular steps (steps with a
local recomputation) and Picard sweeps at every step; time and step size to
1e-12 relative (the two sum the same values in different orders).
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "explosion_masks_81sq_N5.npz")


@pytest.fixture(scope="module")
def eb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import exahype_b200
    exahype_b200.load()
    return exahype_b200


def test_explosion_81x81_mask_every_step_to_t02(eb):
    from exahype_b200 import problems
    ref = np.load(GOLDEN)
    status, t_ref, dt_ref = ref["status"], ref["t"], ref["dt"]
    irr_ref, sw_ref = ref["irregular"], ref["sweeps"]
    nsteps = len(t_ref) - 1
    assert t_ref[-1] >= 0.2 > t_ref[-2] and nsteps > 700

    luh, fv, _ = problems.explosion(2, 5, (81, 81), seed=0)
    s = eb.Solver(2, 5)
    g = eb.LimitingMesh(s, (81, 81), [0.0, 0.0], [1.0, 1.0], eb.BC_OUTFLOW, helper_layers=1, cure_steps=0)
    g.set_solution(luh)
    g.set_fv_initial(fv)
    g.init(0.0)

    def check(k):
        sg = g.status()
        diff = np.nonzero(sg != status[k])[0]
        assert diff.size == 0, "step %d: status differs in %d cells, first %s: gpu %s reference %s" % (
            k, diff.size, diff[:8].tolist(), sg[diff[:8]].tolist(), status[k][diff[:8]].tolist())
        st = g.state()
        assert st["steps"] == k
        assert st["irregular_steps"] == irr_ref[k], (k, st, irr_ref[k])
        assert st["picard_sweeps"] == sw_ref[k], (k, st, sw_ref[k])
        assert abs(st["t"] - t_ref[k]) <= 1e-12 * max(t_ref[k], 1e-300), (k, st["t"], t_ref[k])
        assert abs(st["dt"] - dt_ref[k]) <= 1e-12 * dt_ref[k], (k, st["dt"], dt_ref[k])
        return st

    check(0)
    for k in range(1, nsteps + 1):
        g.step(1)
        st = check(k)
    # the reference's loop ends here too: t >= 0.2 after exactly nsteps steps
    assert st["t"] >= 0.2
    assert (status[-1] == 3).any() and irr_ref[-1] > 0.9 * nsteps
