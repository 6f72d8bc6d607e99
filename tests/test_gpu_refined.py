"""Statically refined meshes (exa_mesh_create_refined) on the GPU against the
oracle's restatement of the reference's hanging-face sequencing
(pyoracle.RefinedMesh over the C kernels): ancestors receive the restriction
of their fine children's face data, descendants the prolongation of their
coarse parent's, Riemann problems pair cells with both.

Bar: solution 1e-12 relative L2 (the restriction's additions run in any
order on the GPU), equal step and Picard sweep counts, time and step size to
1e-13 relative; a constant state stays constant to 1e-10 (the 13-digit
operator tables leave round-off of that order)."""
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


CASES = [(2, 3, (9, 9), (3, 3), (6, 6), 10, 0), (2, 5, (7, 8), (2, 3), (4, 5), 6, 3),
         (3, 3, (4, 4, 4), (1, 1, 1), (2, 2, 2), 4, 0), (3, 5, (5, 5, 5), (2, 2, 2), (3, 3, 3), 3, 2),
         (3, 5, (5, 5, 5), (2, 2, 2), (3, 3, 3), 3, 0), (3, 5, (5, 5, 5), (2, 2, 2), (3, 3, 3), 3, 8)]


@pytest.mark.parametrize("dim,N,cells,lo,hi,steps,variant", CASES)
def test_refined_mesh_vs_oracle(eb, dim, N, cells, lo, hi, steps, variant):
    from exahype_b200 import problems
    u = problems.pulse_refined(dim, N, cells, lo, hi, seed=4)
    s = eb.Solver(dim, N)
    s.variant = variant
    m = eb.Mesh.refined(s, cells, [0.0] * dim, [1.0] * dim, lo, hi)
    o = pyoracle.RefinedMesh(dim, N, cells, [1.0] * dim, lo, hi)
    assert m.ncells == o.ncells == u.shape[0]
    m.set_solution(u)
    o.set_solution(u)
    m.init(0.0)
    o.init(0.0)
    assert m.state()["dt"] == o.state()["dt"]  # from identical data: bit-identical
    m.step(steps)
    o.step(steps)
    a, b = m.get_solution(), o.get_solution()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    sa, sb = m.state(), o.state()
    assert sa["steps"] == sb["steps"] == steps
    assert sa["picard_sweeps"] == sb["picard_sweeps"]
    close = lambda x, y: abs(x - y) <= 1e-13 * abs(y)  # noqa: E731
    assert close(sa["t"], sb["t"]) and close(sa["dt"], sb["dt"])
    # the pulse crossed into and through the refined box
    assert np.linalg.norm(a - u) / np.linalg.norm(u) > 1e-6


@pytest.mark.parametrize("dim,N,cells,lo,hi,steps", [(2, 4, (7, 7), (2, 2), (5, 5), 8),
                                                     (3, 3, (4, 4, 4), (1, 1, 1), (2, 2, 2), 4)])
def test_refined_elastic_mesh_vs_oracle(eb, dim, N, cells, lo, hi, steps):
    """the linear kernels (elastic waves) on a refined mesh"""
    from exahype_b200 import problems
    u = problems.elastic_pulse_refined(dim, N, cells, lo, hi, seed=4)
    s = eb.Solver(dim, N, eb.PDE_ELASTIC)
    m = eb.Mesh.refined(s, cells, [0.0] * dim, [1.0] * dim, lo, hi)
    o = pyoracle.RefinedMesh(dim, N, cells, [1.0] * dim, lo, hi, pde=2)
    m.set_solution(u)
    o.set_solution(u)
    m.init(0.0)
    o.init(0.0)
    assert m.state()["dt"] == o.state()["dt"]
    m.step(steps)
    o.step(steps)
    a, b = m.get_solution(), o.get_solution()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    sa, sb = m.state(), o.state()
    assert sa["steps"] == sb["steps"] == steps
    assert abs(sa["t"] - sb["t"]) <= 1e-13 * sb["t"]


NESTED = [(2, 3, (9, 9), [((3, 3), (6, 6)), ((10, 10), (17, 17))], 8, 0),
          (2, 5, (9, 9), [((3, 3), (6, 6)), ((10, 11), (15, 17)), ((31, 34), (44, 50))], 4, 3),
          (3, 3, (4, 4, 4), [((1, 1, 1), (3, 3, 3)), ((4, 4, 4), (5, 5, 5))], 3, 2)]


@pytest.mark.parametrize("dim,N,cells,boxes,steps,variant", NESTED)
def test_nested_mesh_vs_oracle(eb, dim, N, cells, boxes, steps, variant):
    """nested refined boxes (three and four levels): every level's hanging
    faces through its own ancestors and descendants"""
    from exahype_b200 import problems
    u = problems.pulse_nested(dim, N, cells, boxes, seed=6)
    s = eb.Solver(dim, N)
    s.variant = variant
    m = eb.Mesh.nested(s, cells, [0.0] * dim, [1.0] * dim, boxes)
    o = pyoracle.RefinedMesh(dim, N, cells, [1.0] * dim, boxes=boxes)
    assert m.ncells == o.ncells == u.shape[0]
    m.set_solution(u)
    o.set_solution(u)
    m.init(0.0)
    o.init(0.0)
    assert m.state()["dt"] == o.state()["dt"]
    m.step(steps)
    o.step(steps)
    a, b = m.get_solution(), o.get_solution()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    sa, sb = m.state(), o.state()
    assert sa["steps"] == sb["steps"] == steps
    assert sa["picard_sweeps"] == sb["picard_sweeps"]
    assert abs(sa["t"] - sb["t"]) <= 1e-13 * sb["t"]


def test_nested_mesh_outflow_vs_oracle(eb):
    """outflow domain faces on the coarse level (their boundary Riemann
    problems with the outflow state run every step)"""
    from exahype_b200 import problems
    cells, boxes = (9, 9), [((3, 3), (6, 6)), ((10, 10), (17, 17))]
    u = problems.pulse_nested(2, 3, cells, boxes, seed=6)
    s = eb.Solver(2, 3)
    m = eb.Mesh.nested(s, cells, [0.0, 0.0], [1.0, 1.0], boxes, bc=eb.BC_OUTFLOW)
    o = pyoracle.RefinedMesh(2, 3, cells, [1.0, 1.0], boxes=boxes, bc=0)
    assert len(o.bnd) == 4 * 9
    m.set_solution(u)
    o.set_solution(u)
    m.init(0.0)
    o.init(0.0)
    m.step(10)
    o.step(10)
    a, b = m.get_solution(), o.get_solution()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    assert m.state()["picard_sweeps"] == o.state()["picard_sweeps"]
    with pytest.raises(eb.ExaError):  # periodic on one face of an axis only
        eb.Mesh.nested(s, cells, [0.0, 0.0], [1.0, 1.0], boxes, bc=[-1, 0, 0, 0])


def test_nested_mesh_free_stream_and_arguments(eb):
    s = eb.Solver(2, 3)
    boxes = [((3, 3), (6, 6)), ((10, 10), (17, 17))]
    m = eb.Mesh.nested(s, (9, 9), [0.0, 0.0], [1.0, 1.0], boxes)
    u = np.zeros(m.solution_shape)
    u[..., 0], u[..., 1], u[..., 2], u[..., 4] = 1.0, 0.4, -0.2, 2.5
    m.set_solution(u)
    m.init(0.0)
    m.step(10)
    assert np.abs(m.get_solution() - u).max() < 1e-10
    for bad in ([((3, 3), (6, 6)), ((9, 10), (17, 17))], [((3, 3), (6, 6)), ((10, 10), (18, 17))]):
        with pytest.raises(eb.ExaError):  # the inner box touches its level's region
            eb.Mesh.nested(s, (9, 9), [0.0, 0.0], [1.0, 1.0], bad)


def test_refined_mesh_free_stream(eb):
    s = eb.Solver(2, 5)
    m = eb.Mesh.refined(s, (9, 9), [0.0, 0.0], [1.0, 1.0], (3, 3), (6, 6))
    u = np.zeros(m.solution_shape)
    u[..., 0], u[..., 1], u[..., 2], u[..., 4] = 1.0, 0.4, -0.2, 2.5
    m.set_solution(u)
    m.init(0.0)
    m.step(20)
    assert np.abs(m.get_solution() - u).max() < 1e-10


def test_refined_mesh_arguments(eb):
    s = eb.Solver(2, 3)
    for lo, hi in (((0, 3), (6, 6)), ((3, 3), (9, 6)), ((4, 3), (4, 6))):
        with pytest.raises(eb.ExaError):
            eb.Mesh.refined(s, (9, 9), [0.0, 0.0], [1.0, 1.0], lo, hi)


def test_nested_mesh_write_vtk(eb, tmp_path):
    """both VTK layouts on a nested mesh: every cell's points at its own
    level's position and width"""
    import importlib.util
    import os
    from exahype_b200 import problems
    spec = importlib.util.spec_from_file_location("amr_t", os.path.join(os.path.dirname(__file__), "test_gpu_amr.py"))
    amr_t = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(amr_t)
    cells, boxes = (9, 9), [((3, 3), (6, 6)), ((10, 10), (17, 17))]
    s = eb.Solver(2, 3)
    m = eb.Mesh.nested(s, cells, [0.0, 0.0], [1.0, 1.0], boxes)
    u = problems.pulse_nested(2, 3, cells, boxes, seed=6)
    m.set_solution(u)
    m.init(0.0)
    m.step(2)
    sol = m.get_solution()
    path = str(tmp_path / "nested_l.vtk")
    m.write_vtk_legendre(path, binary=True)
    v = amr_t.read_vtk(path)
    X = problems.nested_node_coordinates(2, 3, cells, boxes).reshape(-1, 2)
    assert np.allclose(v["points"][:, :2], X, rtol=0, atol=1e-14)
    assert np.array_equal(v["Q"], sol.reshape(-1, 5))
    path = str(tmp_path / "nested_c.vtk")
    m.write_vtk(path)
    v = amr_t.read_vtk(path)
    ref_q = np.concatenate([pyoracle.plot_vertices(2, 3, 5, sol[c]).reshape(-1, 5) for c in range(m.ncells)])
    assert np.max(np.abs(v["Q"] - ref_q)) <= 1e-12 * np.max(np.abs(ref_q))
    assert np.allclose(v["points"].min(axis=0)[:2], 0.0) and np.allclose(v["points"].max(axis=0)[:2], 1.0)


@pytest.mark.parametrize("boxes,w", [([((3, 3), (6, 6))], 0.99), ([((3, 3), (6, 6)), ((10, 10), (17, 17))], 0.9)])
def test_nested_mesh_fused_vs_oracle(eb, boxes, w):
    """fused time stepping on refined meshes: the predictor of every level
    runs right after the update with the estimated step, rerun with
    weight * stable when the estimate was too large"""
    from exahype_b200 import problems
    cells = (9, 9)
    u = problems.pulse_nested(2, 3, cells, boxes, seed=8)
    s = eb.Solver(2, 3)
    m = eb.Mesh.nested(s, cells, [0.0, 0.0], [1.0, 1.0], boxes)
    o = pyoracle.RefinedMesh(2, 3, cells, [1.0, 1.0], boxes=boxes)
    m.set_solution(u)
    o.set_solution(u)
    m.init_fused(0.0, w)
    o.init_fused(0.0, w)
    m.step(12)
    o.step(12)
    a, b = m.get_solution(), o.get_solution()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    sa, sb = m.state(), o.state()
    assert sa["steps"] == sb["steps"] == 12 and sa["picard_sweeps"] == sb["picard_sweeps"]
    close = lambda x, y: abs(x - y) <= 1e-13 * abs(y)  # noqa: E731
    assert close(sa["t"], sb["t"]) and close(sa["dt"], sb["dt"])
    fa, fb = m.fused_state(), o.fused_state()
    assert close(fa["predictor_dt"], fb["predictor_dt"]) and fa["reruns"] == fb["reruns"]


BOXES = [(2, 3, (12, 12), [(0, (2, 2), (5, 5)), (0, (7, 6), (10, 10)), (1, (8, 8), (12, 12))], 6, 0, -1),
         (2, 5, (12, 9), [(0, (2, 2), (5, 4)), (0, (5, 2), (7, 7)), (0, (8, 3), (10, 6))], 4, 2, 0),
         (3, 3, (6, 5, 5), [(0, (1, 1, 1), (3, 3, 3)), (0, (3, 2, 2), (5, 4, 4))], 3, 6, -1)]


@pytest.mark.parametrize("dim,N,cells,boxes,steps,variant,bc", BOXES)
def test_boxes_mesh_vs_oracle(eb, dim, N, cells, boxes, steps, variant, bc):
    """several refined boxes per level (disjoint, touching and overlapping:
    their union is refined), one level refined again, outflow or periodic"""
    from exahype_b200 import problems
    u = problems.pulse_boxes(dim, N, cells, boxes, seed=9)
    s = eb.Solver(dim, N)
    s.variant = variant
    m = eb.Mesh.boxes(s, cells, [0.0] * dim, [1.0] * dim, boxes, bc=bc)
    o = pyoracle.RefinedMesh(dim, N, cells, [1.0] * dim, level_boxes=boxes, bc=bc)
    assert m.ncells == o.ncells == u.shape[0]
    m.set_solution(u)
    o.set_solution(u)
    m.init(0.0)
    o.init(0.0)
    assert m.state()["dt"] == o.state()["dt"]
    m.step(steps)
    o.step(steps)
    a, b = m.get_solution(), o.get_solution()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    sa, sb = m.state(), o.state()
    assert sa["steps"] == sb["steps"] == steps and sa["picard_sweeps"] == sb["picard_sweeps"]
    assert abs(sa["t"] - sb["t"]) <= 1e-13 * sb["t"]


def test_boxes_mesh_arguments(eb):
    s = eb.Solver(2, 3)
    for boxes in ([(0, (0, 2), (5, 5))],                       # no margin to the domain
                  [(0, (2, 2), (5, 5)), (1, (6, 6), (9, 9))],  # no margin inside level 1
                  [(1, (8, 8), (12, 12))],                     # level 1 has no region
                  [(0, (3, 3), (3, 5))]):                      # empty
        with pytest.raises(eb.ExaError):
            eb.Mesh.boxes(s, (12, 12), [0.0, 0.0], [1.0, 1.0], boxes)


@pytest.mark.parametrize("boxes,bc", [([], [1, 1, 1, 1]), ([], [1, 1, 0, 0]),
                                      ([(0, (2, 2), (5, 5)), (1, (7, 7), (13, 13))], [1, 1, 1, 1])])
def test_reflective_walls_vs_oracle(eb, boxes, bc):
    """reflective walls (the reference demonstrator's boundaryValues: normal
    momentum negated) on a uniform mesh and on a refined one, against the
    oracle's restatement; a density and pressure pulse at rest, so that the
    walls see acoustic waves, not a flow driven into them"""
    from exahype_b200 import problems
    cells = (9, 9)
    s = eb.Solver(2, 3)
    if boxes:
        u = problems.pulse_boxes(2, 3, cells, boxes, seed=10)
        m = eb.Mesh.boxes(s, cells, [0.0, 0.0], [1.0, 1.0], boxes, bc=bc)
    else:
        u, _ = problems.gaussian_pulse_2d(3, cells, seed=10)
        m = eb.Mesh(s, cells, [0.0, 0.0], [1.0, 1.0], bc)
    u[..., 1:4] = 0.0
    u[..., 4] = u[..., 0] / 0.4  # p = rho
    o = pyoracle.RefinedMesh(2, 3, cells, [1.0, 1.0], level_boxes=boxes, bc=bc)
    assert m.ncells == o.ncells
    m.set_solution(u)
    o.set_solution(u)
    m.init(0.0)
    o.init(0.0)
    m.step(15)
    o.step(15)
    a, b = m.get_solution(), o.get_solution()
    assert np.isfinite(b).all()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    assert m.state()["picard_sweeps"] == o.state()["picard_sweeps"]


@pytest.mark.parametrize("dim,N,cells,seq", [
    (2, 3, (9, 9), [[(0, (3, 3), (6, 6))], [(0, (4, 3), (7, 7)), (1, (13, 11), (18, 17))], [],
                    [(0, (2, 2), (8, 5))]]),
    (3, 3, (5, 5, 5), [[], [(0, (1, 1, 1), (3, 3, 3))], [(0, (2, 2, 2), (4, 4, 4)), (1, (7, 7, 7), (11, 10, 10))]])])
def test_regrid_vs_oracle(eb, dim, N, cells, seq):
    """static AMR between steps: refine, move, coarsen and refine twice;
    every transfer (copy, prolongation over one or two levels, restriction
    of one or two finer levels) against the oracle's restatement"""
    from exahype_b200 import problems
    s = eb.Solver(dim, N)
    u = problems.pulse_boxes(dim, N, cells, seq[0], seed=12) if seq[0] else \
        (problems.gaussian_pulse_2d(N, cells, seed=12)[0] if dim == 2 else problems.gaussian_pulses_3d(N, cells, seed=12)[0])
    m = eb.Mesh.boxes(s, cells, [0.0] * dim, [1.0] * dim, seq[0])
    o = pyoracle.RefinedMesh(dim, N, cells, [1.0] * dim, level_boxes=seq[0])
    m.set_solution(u)
    o.set_solution(u)
    m.init(0.0)
    o.init(0.0)
    close = lambda x, y: abs(x - y) <= 1e-13 * abs(y)  # noqa: E731
    for boxes in seq[1:] + [seq[0]]:
        m.step(2)
        o.step(2)
        m.regrid(boxes)
        o.regrid(boxes)
        assert m.ncells == o.ncells
        a, b = m.get_solution(), o.get_solution()
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
        sa, sb = m.state(), o.state()
        assert sa["steps"] == sb["steps"] and sa["picard_sweeps"] == sb["picard_sweeps"]
        assert close(sa["t"], sb["t"]) and close(sa["dt"], sb["dt"])


def test_regrid_keeps_a_constant_state(eb):
    s = eb.Solver(2, 5)
    m = eb.Mesh.boxes(s, (9, 9), [0.0, 0.0], [1.0, 1.0], [])
    u = np.zeros(m.solution_shape)
    u[..., 0], u[..., 1], u[..., 4] = 1.0, 0.3, 2.5
    m.set_solution(u)
    m.init(0.0)
    for boxes in ([(0, (3, 3), (6, 6)), (1, (10, 10), (17, 17))], [(0, (2, 4), (5, 7))], []):
        m.regrid(boxes)
        m.step(1)
        v = m.get_solution()
        assert np.abs(v[..., 0] - 1.0).max() < 1e-10 and np.abs(v[..., 1] - 0.3).max() < 1e-10
    with pytest.raises(eb.ExaError):
        m.regrid([(0, (0, 0), (3, 3))])  # no margin
    assert m.validate() == 0


def test_adaptive_refinement_loop_vs_oracle(eb):
    """a refinement criterion (density variation within a cell: REFINE above
    2 %, ERASE below 0.5 %, KEEP between) drives adapt_boxes and regrid
    between steps; the oracle follows the same boxes"""
    from exahype_b200 import problems
    cells = (9, 9)
    u, _ = problems.gaussian_pulse_2d(3, cells, seed=13)
    s = eb.Solver(2, 3)
    m = eb.Mesh.boxes(s, cells, [0.0, 0.0], [1.0, 1.0], [])
    o = pyoracle.RefinedMesh(2, 3, cells, [1.0, 1.0], level_boxes=[])
    m.set_solution(u)
    o.set_solution(u)
    m.init(0.0)
    o.init(0.0)
    refined_once = False
    for _ in range(3):
        v = m.get_solution()[..., 0]
        var = (v.max(axis=1) - v.min(axis=1)) / v.mean(axis=1)
        controls = np.where(var > 0.02, eb.REFINE, np.where(var < 0.005, eb.ERASE, eb.KEEP))
        boxes = eb.adapt_boxes(m, controls, 2)
        refined_once |= bool(boxes)
        m.regrid(boxes)
        o.regrid(boxes)
        m.step(2)
        o.step(2)
        a, b = m.get_solution(), o.get_solution()
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
        assert m.validate() == 0
    assert refined_once and m.ncells > 81
