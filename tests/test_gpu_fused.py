"""Fused time stepping (exa_mesh_init_fused) on the GPU against the oracle
harness's restatement of the reference's fused scheme (oracle/harness.c
hrn_step_fused): predictor right after the update with the estimated step,
rerun with weight * stable when the estimate was too large.

Bar: solution 1e-12 relative L2; step and rerun counts identical; corrector
time stamp and step size and the predictor step estimate to 1e-14 relative
(the bookkeeping runs in round-to-nearest arithmetic on both sides, but the
stable step of solutions that differ at round-off can differ in its last
bit)."""
import numpy as np
import pytest

import pyoracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import exahype_b200
    exahype_b200.load()
    return exahype_b200


CASES = [(2, 3, (12, 12), -1, 0, 30, 0.99), (2, 5, (8, 8), 0, 0, 20, 0.9), (3, 3, (5, 5, 5), -1, 0, 10, 0.99),
         (3, 5, (4, 4, 4), -1, 0, 8, 0.99), (2, 4, (8, 8), -1, 2, 15, 0.95)]
# predictor variants of the nonlinear cases: 0 (node form), 1, 2, 6, 7 (line
# forms), 8 (line form, iterate in tensor memory), 5 (mixed precision); the
# rerun launch is gated by a device count
VARIANTS = [0, 1, 2, 5, 6, 7, 8]


def _params():
    out = []
    for c in CASES:
        for v in (VARIANTS if c[4] != 2 else [0]):
            out.append(c + (v,))
    return out


@pytest.mark.parametrize("dim,N,cells,bc,pde,steps,w,variant", _params())
def test_fused_mesh_vs_oracle(eb, dim, N, cells, bc, pde, steps, w, variant):
    from exahype_b200 import problems
    if pde == 2:
        u, _ = problems.elastic_pulse(dim, N, cells, seed=2)
    elif dim == 2:
        u, _ = problems.gaussian_pulse_2d(N, cells, seed=2)
    else:
        u, _ = problems.gaussian_pulses_3d(N, cells, seed=2)
    s = eb.Solver(dim, N, pde)
    s.variant = variant
    m = eb.Mesh(s, cells, [0.0] * dim, [1.0] * dim, bc)
    m.set_solution(u)
    m.init_fused(0.0, w)
    m.step(steps)
    o = pyoracle.Mesh(dim, N, cells, [1.0] * dim, bc, pde=pde, nthreads=8)
    o.set_solution(u)
    o.init_fused(0.0, w)
    o.step(steps)
    a, b = m.get_solution(), o.get_solution()
    # mixed variant: FP32 increments in the Picard sweeps (1e-9 bar)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < (1e-9 if variant == 5 else 1e-12)
    sa, sb = m.state(), o.state()
    assert sa["steps"] == sb["steps"] == steps
    # the stable step of a solution that differs at round-off may differ in
    # its last bit, and the time stamp sums the steps
    tol = 1e-11 if variant == 5 else 1e-14
    close = lambda x, y: abs(x - y) <= tol * abs(y)
    assert close(sa["t"], sb["t"]) and close(sa["dt"], sb["dt"])
    fa, fb = m.fused_state(), o.fused_state()
    assert close(fa["predictor_dt"], fb["predictor_dt"]) and fa["reruns"] == fb["reruns"]
    if pde != 2 and variant != 5:
        assert sa["picard_sweeps"] == sb["picard_sweeps"]
    # run_until stops on the same step
    t_end = sa["t"] + 4.5 * sa["dt"]
    assert m.run_until(t_end) == o.run_until(t_end)
    assert close(m.state()["t"], o.state()["t"])


def test_fused_first_step_equals_unfused(eb):
    """the first fused step updates with the initial data's stable step and
    the predictor computed with it, like the non-fused scheme; the fused
    state of a non-fused mesh is an error"""
    from exahype_b200 import problems
    u, _ = problems.gaussian_pulse_2d(3, (12, 12), seed=2)
    s = eb.Solver(2, 3)
    f = eb.Mesh(s, (12, 12), [0, 0], [1, 1], eb.BC_PERIODIC)
    f.set_solution(u)
    f.init_fused(0.0, 0.99)
    f.step(1)
    assert f.fused_state()["reruns"] >= 0
    n = eb.Mesh(s, (12, 12), [0, 0], [1, 1], eb.BC_PERIODIC)
    n.set_solution(u)
    n.init(0.0)
    n.step(1)
    # same first corrector step size (both start from the initial data's)
    a, b = f.get_solution(), n.get_solution()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    with pytest.raises(eb.ExaError):
        n.fused_state()
