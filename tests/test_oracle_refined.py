"""The oracle's refined-mesh sequencing (pyoracle.RefinedMesh) run over the
C restatement and over the reference's kernels compiled from its sources
(oracle/_ref, when present): the same fields to 1e-12 relative L2, the same
step and Picard sweep counts; a constant state stays constant."""
import numpy as np
import pytest

import pyoracle


@pytest.mark.parametrize("dim,N,cells,lo,hi,steps", [(2, 3, (9, 9), (3, 3), (6, 6), 4),
                                                     (3, 3, (4, 4, 4), (1, 1, 1), (2, 2, 2), 2)])
def test_refined_oracle_vs_reference_kernels(dim, N, cells, lo, hi, steps):
    if not pyoracle.ref_available(dim):
        pytest.skip("compiled reference kernels not built")
    from exahype_b200 import problems
    u = problems.pulse_refined(dim, N, cells, lo, hi, seed=4)
    res = []
    for impl in ("oracle", "ref"):
        m = pyoracle.RefinedMesh(dim, N, cells, [1.0] * dim, lo, hi, impl=impl)
        m.set_solution(u)
        m.init(0.0)
        m.step(steps)
        res.append((m.get_solution(), m.state()))
    (a, sa), (b, sb) = res
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    assert sa["steps"] == sb["steps"] and sa["picard_sweeps"] == sb["picard_sweeps"]
    assert abs(sa["t"] - sb["t"]) <= 1e-13 * sb["t"]


def test_refined_oracle_elastic_vs_reference_kernels():
    if not pyoracle.ref_available(2):
        pytest.skip("compiled reference kernels not built")
    from exahype_b200 import problems
    cells, lo, hi = (7, 7), (2, 2), (5, 5)
    u = problems.elastic_pulse_refined(2, 4, cells, lo, hi, seed=4)
    res = []
    for impl in ("oracle", "ref"):
        m = pyoracle.RefinedMesh(2, 4, cells, [1.0, 1.0], lo, hi, pde=2, impl=impl)
        m.set_solution(u)
        m.init(0.0)
        m.step(3)
        res.append(m.get_solution())
    assert np.linalg.norm(res[0] - res[1]) / np.linalg.norm(res[1]) < 1e-12


def test_nested_oracle_vs_reference_kernels():
    if not pyoracle.ref_available(2):
        pytest.skip("compiled reference kernels not built")
    from exahype_b200 import problems
    cells, boxes = (9, 9), [((3, 3), (6, 6)), ((10, 10), (17, 17))]
    u = problems.pulse_nested(2, 3, cells, boxes, seed=6)
    res = []
    for impl in ("oracle", "ref"):
        m = pyoracle.RefinedMesh(2, 3, cells, [1.0, 1.0], boxes=boxes, impl=impl)
        m.set_solution(u)
        m.init(0.0)
        m.step(3)
        res.append((m.get_solution(), m.state()))
    (a, sa), (b, sb) = res
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    assert sa["picard_sweeps"] == sb["picard_sweeps"]


def test_boxes_oracle_vs_reference_kernels():
    if not pyoracle.ref_available(2):
        pytest.skip("compiled reference kernels not built")
    from exahype_b200 import problems
    cells, boxes = (12, 12), [(0, (2, 2), (5, 5)), (0, (7, 6), (10, 10)), (1, (8, 8), (12, 12))]
    u = problems.pulse_boxes(2, 3, cells, boxes, seed=9)
    res = []
    for impl in ("oracle", "ref"):
        m = pyoracle.RefinedMesh(2, 3, cells, [1.0, 1.0], level_boxes=boxes, impl=impl)
        m.set_solution(u)
        m.init(0.0)
        m.step(2)
        res.append(m.get_solution())
    assert np.linalg.norm(res[0] - res[1]) / np.linalg.norm(res[1]) < 1e-12


def test_regrid_oracle_vs_reference_kernels():
    """the regrid transfers through the C restatement's and the reference's
    compiled amrRoutines agree"""
    if not pyoracle.ref_available(2):
        pytest.skip("compiled reference kernels not built")
    from exahype_b200 import problems
    b1, b2 = [(0, (3, 3), (6, 6))], [(0, (4, 3), (7, 7)), (1, (13, 11), (18, 17))]
    u = problems.pulse_boxes(2, 3, (9, 9), b1, seed=12)
    res = []
    for impl in ("oracle", "ref"):
        m = pyoracle.RefinedMesh(2, 3, (9, 9), [1.0, 1.0], level_boxes=b1, impl=impl)
        m.set_solution(u)
        m.init(0.0)
        m.step(1)
        m.regrid(b2)
        m.step(1)
        m.regrid([])
        res.append(m.get_solution())
    assert np.linalg.norm(res[0] - res[1]) / np.linalg.norm(res[1]) < 1e-12


def test_refined_oracle_free_stream():
    m = pyoracle.RefinedMesh(2, 3, (9, 9), [1.0, 1.0], (3, 3), (6, 6))
    u = np.zeros((m.ncells, 16, 5))
    u[..., 0], u[..., 1], u[..., 4] = 1.0, 0.3, 2.5
    m.set_solution(u)
    m.init(0.0)
    m.step(3)
    assert np.abs(m.get_solution() - u).max() < 1e-10


def test_refined_oracle_elastic_walls_vs_reference_kernels():
    """the linear kernels' boundary faces on a refined mesh: rigid walls in x,
    outflow in y"""
    if not pyoracle.ref_available(2):
        pytest.skip("compiled reference kernels not built")
    from exahype_b200 import problems
    cells, lo, hi = (7, 7), (2, 2), (5, 5)
    u = problems.elastic_pulse_refined(2, 3, cells, lo, hi, seed=4)
    res = []
    for impl in ("oracle", "ref"):
        m = pyoracle.RefinedMesh(2, 3, cells, [1.0, 1.0], lo, hi, pde=2, impl=impl, bc=[1, 1, 0, 0])
        m.set_solution(u)
        m.init(0.0)
        m.step(4)
        res.append(m.get_solution())
    assert np.linalg.norm(res[0] - res[1]) / np.linalg.norm(res[1]) < 1e-12
