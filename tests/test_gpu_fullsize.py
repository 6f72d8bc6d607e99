"""The benchmark workloads at their full sizes, on the GPU through the C ABI.

* The 3D Euler N=5 27^3 periodic pulses workload (21.3 M degrees of freedom,
  seed 0, as the benchmark runs it) for its full 20 time steps against the
  oracle run with all host threads (about 10 s on 16 threads): the FP64
  predictor to 1e-12 relative L2 with equal step and Picard sweep counts,
  the mixed-precision predictor (both register budgets) to 1e-9 relative L2
  with the same step count; times to 1e-12 relative.
* The 3D elastic-wave N=5 mesh of the same size (38.3 M): two steps against
  the oracle, fields to 1e-12 relative L2, the first step size bit-identical
  (later ones to 1e-14: they come from solutions that differ at round-off).
  The Euler mesh the same way with seed 7.
* Size-independent property of the Euler mesh over 20 steps: with periodic
  boundaries the Rusanov flux of every face enters both cells with opposite
  signs and the stiffness terms integrate the constant test function to zero,
  so the quadrature-weighted total of every conserved variable stays constant
  up to round-off (bound: 1e-12 of the total of absolute values).

The 81 x 81 limiter workload is covered at full size in test_gpu_limiter.py.
"""
import os

import numpy as np
import pytest

import pyoracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CELLS = (27, 27, 27)


@pytest.fixture(scope="module")
def eb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import exahype_b200
    exahype_b200.load()
    return exahype_b200


C1_STEPS = 20


@pytest.fixture(scope="module")
def c1_oracle():
    """the oracle's 20 steps of the benchmark workload (seed 0)"""
    from exahype_b200 import problems
    u = problems.gaussian_pulses_3d(5, CELLS, seed=0)[0]
    o = pyoracle.Mesh(3, 5, CELLS, [1.0] * 3, -1, nthreads=os.cpu_count() or 1)
    o.set_solution(u)
    o.init(0.0)
    dt0 = o.state()["dt"]
    o.step(C1_STEPS)
    return u, dt0, o.get_solution(), o.state()


@pytest.mark.parametrize("variant,tol", [(2, 1e-12), (0, 1e-12), (6, 1e-12), (8, 1e-12), (4, 1e-9), (5, 1e-9)])
def test_benchmark_workload_20_steps_vs_oracle(eb, c1_oracle, variant, tol):
    """variants: 0 the node form, 2 and 6 line forms, 8 the line form with the
    iterate in tensor memory (the benchmark runs the autotuner's choice among
    them), 4 and 5 the mixed-precision line form"""
    u, dt0, exp, st = c1_oracle
    s = eb.Solver(3, 5, eb.PDE_EULER)
    s.variant = variant
    m = eb.Mesh(s, CELLS, [0.0] * 3, [1.0] * 3, eb.BC_PERIODIC)
    m.set_solution(u)
    m.init(0.0)
    assert m.state()["dt"] == dt0  # from identical data: bit-identical
    m.step(C1_STEPS)
    got = m.get_solution()
    err = np.linalg.norm(got - exp) / np.linalg.norm(exp)
    assert err <= tol, "variant %d: relative L2 %.3e after %d steps" % (variant, err, C1_STEPS)
    a = m.state()
    assert a["steps"] == st["steps"] == C1_STEPS
    assert abs(a["t"] - st["t"]) <= 1e-12 * st["t"]
    if tol <= 1e-12:
        assert a["picard_sweeps"] == st["picard_sweeps"]
    else:
        assert abs(a["picard_sweeps"] - st["picard_sweeps"]) <= 0.02 * st["picard_sweeps"]


def _initial(pde, order):
    from exahype_b200 import problems
    if pde == 2:
        return problems.elastic_pulse(3, order, CELLS, seed=7)[0]
    return problems.gaussian_pulses_3d(order, CELLS, seed=7)[0]


@pytest.mark.parametrize("pde", [0, 2])
def test_full_size_two_steps_vs_oracle(eb, pde):
    u = _initial(pde, 5)
    s = eb.Solver(3, 5, pde)
    if pde == 0:
        s.variant = 2  # the line form the benchmark runs
    m = eb.Mesh(s, CELLS, [0.0] * 3, [1.0] * 3, eb.BC_PERIODIC)
    m.set_solution(u)
    m.init(0.0)
    o = pyoracle.Mesh(3, 5, CELLS, [1.0] * 3, eb.BC_PERIODIC, pde=pde, nthreads=os.cpu_count() or 1)
    o.set_solution(u)
    o.init(0.0)
    # the first step size comes from identical data: bit-identical
    assert m.state()["dt"] == o.state()["dt"]
    m.step(2)
    o.step(2)
    a, b = m.get_solution(), o.get_solution()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    sa, sb = m.state(), o.state()
    assert sa["steps"] == sb["steps"] == 2
    # later steps come from solutions that differ at round-off
    assert abs(sa["dt"] - sb["dt"]) <= 1e-14 * sb["dt"]
    assert sa["picard_sweeps"] == sb["picard_sweeps"]


def test_full_size_euler_conservation(eb):
    order = 5
    u = _initial(0, order)
    b = order + 1
    x, w = np.polynomial.legendre.leggauss(b)
    w = w / 2.0  # unit interval
    wn = np.einsum("i,j,k->ijk", w, w, w).reshape(-1)  # node (z, y, x), x fastest
    s = eb.Solver(3, order, eb.PDE_EULER)
    s.variant = 2
    m = eb.Mesh(s, CELLS, [0.0] * 3, [1.0] * 3, eb.BC_PERIODIC)
    m.set_solution(u)
    m.init(0.0)
    u0 = m.get_solution()
    tot0 = np.einsum("p,cpv->v", wn, u0)
    scale = np.einsum("p,cpv->v", wn, np.abs(u0))
    m.step(20)
    u1 = m.get_solution()
    assert np.isfinite(u1).all()
    tot1 = np.einsum("p,cpv->v", wn, u1)
    assert (np.abs(tot1 - tot0) <= 1e-12 * scale).all(), (tot1 - tot0) / scale
    # the solution moved: the pulses are advected
    assert np.linalg.norm(u1 - u0) / np.linalg.norm(u0) > 1e-5
