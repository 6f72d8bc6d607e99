"""The mixed-precision predictor (variants EXA_PREDICTOR_MIXED / _MIXED_2:
FP32 increment sweeps after the first FP64 sweep) against the FP64 oracle:
relative L2 error of the solution at most 1e-9 after 20 steps, the same
number of steps to the same time, and Picard sweep counts within a few per
cent of the FP64 path's."""
import numpy as np
import pytest

import pyoracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-9


@pytest.fixture(scope="module")
def eb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import exahype_b200
    exahype_b200.load()
    return exahype_b200


def case(dim, order, cells, seed):
    from exahype_b200 import problems
    if dim == 2:
        return problems.gaussian_pulse_2d(order, cells, seed=seed)[0]
    return problems.gaussian_pulses_3d(order, cells, seed=seed)[0]


@pytest.mark.parametrize("variant", [4, 5])
@pytest.mark.parametrize("dim,order,cells,steps", [
    (2, 3, (16, 16), 20), (2, 5, (12, 12), 20), (2, 7, (8, 8), 20),
    (3, 3, (8, 8, 8), 20), (3, 5, (7, 7, 7), 20),
])
def test_mixed_vs_fp64_oracle(eb, dim, order, cells, steps, variant):
    u0 = case(dim, order, cells, seed=dim * 10 + order)
    s = eb.Solver(dim, order)
    s.variant = variant
    m = eb.Mesh(s, cells, [0.0] * dim, [1.0] * dim, eb.BC_PERIODIC)
    m.set_solution(u0)
    m.init(0.0)
    m.step(steps)
    got = m.get_solution()
    o = pyoracle.Mesh(dim, order, cells, [1.0] * dim, -1, nthreads=8)
    o.set_solution(u0)
    o.init(0.0)
    o.step(steps)
    exp = o.get_solution()
    err = np.linalg.norm(got - exp) / np.linalg.norm(exp)
    assert err <= TOL, "mixed predictor: relative L2 %.3e" % err
    a, b = m.state(), o.state()
    assert a["steps"] == b["steps"]
    assert abs(a["t"] - b["t"]) <= 1e-9 * b["t"]
    assert abs(a["picard_sweeps"] - b["picard_sweeps"]) <= 0.05 * b["picard_sweeps"]


def test_mixed_variants_are_selectable_not_autotuned(eb):
    s = eb.Solver(3, 5)
    chosen, ms = s.autotune(256)
    assert chosen in (0, 1, 2, 3, 6, 7, 8) and len(ms) == 9 and ms[4] == ms[5] == -1.0
    s.variant = eb.PREDICTOR_MIXED_2
    assert s.variant == 5
