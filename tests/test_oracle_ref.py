"""The C oracle against the reference's own kernels compiled from source
(oracle/_ref): per-kernel and over whole uniform-mesh runs. Skipped where the
reference build is absent."""
import numpy as np
import pytest

import pyoracle
from exahype_b200 import problems

pytestmark = pytest.mark.skipif(not (pyoracle.ref_available(2) and pyoracle.ref_available(3)),
                                reason="oracle/_ref not built")


def rand_cell(rng, P, nD):
    u = np.zeros((P, nD))
    u[:, 0] = 1 + 0.3 * rng.random(P)
    u[:, 1:4] = 0.4 * (rng.random((P, 3)) - 0.5)
    u[:, 4] = 2.5 + 0.5 * rng.random(P)
    return u


@pytest.mark.parametrize("dim,N,pde", [(2, 3, 0), (2, 5, 0), (2, 7, 0), (3, 3, 0), (3, 5, 0), (3, 7, 0), (2, 3, 1),
                                       (3, 3, 1)])
def test_kernels_vs_reference(dim, N, pde):
    rng = np.random.default_rng(dim * 10 + N + 100 * pde)
    o, r = pyoracle.Kernels(dim, N, pde), pyoracle.Kernels(dim, N, pde, impl="ref")
    u = rand_cell(rng, (N + 1) ** dim, 5 + pde)
    dx = [0.05] * dim
    a, b = o.predictor(u, dx, 1e-3, temps=True), r.predictor(u, dx, 1e-3, temps=True)
    assert a["iterations"] == b["iterations"]
    for k in ("lQhbnd", "lFhbnd", "lduh", "lQi", "lFi", "lQhi", "lFhi"):
        assert np.max(np.abs(a[k] - b[k])) <= 1e-13 * max(np.max(np.abs(b[k])), 1.0), k
    assert o.stable_dt(u, dx) == r.stable_dt(u, dx)  # bit-identical time step


@pytest.mark.parametrize("dim,N,cells,steps,bc", [(2, 3, (9, 9), 8, -1), (3, 3, (4, 4, 4), 3, -1),
                                                  (2, 5, (6, 6), 4, 0), (3, 5, (3, 3, 3), 2, -1)])
def test_mesh_vs_reference(dim, N, cells, steps, bc):
    if dim == 2:
        u, _ = problems.gaussian_pulse_2d(N, cells, seed=3)
    else:
        u, _ = problems.gaussian_pulses_3d(N, cells, seed=3)
    res = []
    for impl in ("oracle", "ref"):
        m = pyoracle.Mesh(dim, N, cells, [1.0] * dim, bc, impl=impl, nthreads=4)
        m.set_solution(u)
        m.init(0.0)
        m.step(steps)
        res.append((m.get_solution(), m.state()))
    (a, sa), (b, sb) = res
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-13
    assert sa["picard_sweeps"] == sb["picard_sweeps"]
    assert sa["steps"] == sb["steps"] == steps


@pytest.mark.parametrize("dim,N,cells,steps", [(2, 5, (16, 16), 40), (2, 3, (20, 20), 30), (3, 3, (6, 6, 6), 8)])
def test_limiting_mesh_vs_reference(dim, N, cells, steps):
    """The limiting harness over the C restatement vs over the reference's own
    Limiter.cpp / MUSCL-Hancock / FV halo kernels: identical troubled-cell
    mask at every step, fields to 1e-13."""
    u, fv, _ = problems.explosion(dim, N, cells, seed=1)
    res = []
    for cls in (pyoracle.LimitingMesh, pyoracle.RefLimitingMesh):
        m = cls(dim, N, cells, (1.0,) * dim, 0)
        m.set_solution(u)
        m.set_fv_initial(fv)
        m.init(0.0)
        masks = []
        for _ in range(steps):
            m.step(1)
            masks.append(m.status().copy())
        res.append((m.get_solution(), np.array(masks), m.state()))
    (a, ma, sa), (b, mb, sb) = res
    assert np.array_equal(ma, mb)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-13
    assert abs(sa["t"] - sb["t"]) <= 1e-13 * sb["t"] and sa["irregular_steps"] == sb["irregular_steps"]
    assert (ma >= 3).any()  # the limiter was active


@pytest.mark.parametrize("dim,N,cells,steps", [(2, 3, (9, 9), 12), (3, 3, (4, 4, 4), 4)])
def test_fused_mesh_vs_reference(dim, N, cells, steps):
    """fused time stepping over the C restatement vs over the reference's own
    kernels (the fused sequencing is the harness's, hrn_step_fused)"""
    if dim == 2:
        u, _ = problems.gaussian_pulse_2d(N, cells, seed=3)
    else:
        u, _ = problems.gaussian_pulses_3d(N, cells, seed=3)
    res = []
    for impl in ("oracle", "ref"):
        m = pyoracle.Mesh(dim, N, cells, [1.0] * dim, -1, impl=impl, nthreads=4)
        m.set_solution(u)
        m.init_fused(0.0, 0.99)
        m.step(steps)
        res.append((m.get_solution(), m.state(), m.fused_state()))
    (a, sa, fa), (b, sb, fb) = res
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-13
    assert sa["picard_sweeps"] == sb["picard_sweeps"] and sa["steps"] == sb["steps"] == steps
    assert fa["reruns"] == fb["reruns"] and fa["reruns"] >= 1
    assert abs(sa["t"] - sb["t"]) <= 1e-13 * sb["t"]


@pytest.mark.parametrize("dim,N", [(2, 3), (2, 5), (3, 3), (3, 5)])
def test_boundary_kinds_vs_reference(dim, N):
    """boundary faces of the demonstrator's Euler PDE against the reference's
    kernels: the FV ghost layers of every boundary face for outflow and
    reflective walls (boundaryLayerExtraction + boundaryConditions +
    ghostLayerFillingAtBoundary, bit for bit, the 3D y- and z-left faces
    included, where the reference's extraction repeats the first interior
    layer), and the DG boundary face with reflective walls (boundaryConditions
    + riemannSolverNonlinear)"""
    rng = np.random.default_rng(dim * 11 + N)
    o, r = pyoracle.Kernels(dim, N, 0), pyoracle.Kernels(dim, N, 0, impl="ref")
    E = 2 * N + 1 + 4
    lim = rng.normal(size=E ** dim * 5)
    for face in range(2 * dim):
        for kind in (0, 1):
            assert np.array_equal(o.fv_boundary(lim, face, kind), r.fv_boundary(lim, face, kind)), (face, kind)
    F = (N + 1) ** (dim - 1)
    Q = np.zeros((F, 5))
    Q[:, 0] = 1 + 0.2 * rng.random(F)
    Q[:, 1:4] = 0.3 * (rng.random((F, 3)) - 0.5)
    Q[:, 4] = 2.5 + rng.random(F)
    FIn = rng.normal(size=F * 5)
    for face in range(2 * dim):
        a, b = o.boundary_face(FIn, Q, face, kind=1), r.boundary_face(FIn, Q, face, kind=1)
        assert np.max(np.abs(a - b)) <= 1e-14 * np.max(np.abs(b))


@pytest.mark.parametrize("dim,N,cells,bc,steps", [(2, 5, (12, 12), 1, 30), (2, 3, (14, 10), [1, 1, 0, 0], 30),
                                                  (3, 3, (4, 4, 4), 1, 6), (3, 3, (4, 4, 4), 0, 6)])
def test_limiting_mesh_boundaries_vs_reference(dim, N, cells, bc, steps):
    """a wide explosion whose front reaches every domain face, with reflective
    walls (the demonstrator's DG and FV boundaryValues) or outflow: identical
    troubled-cell masks at every step, fields to 1e-13"""
    u, fv, _ = problems.explosion(dim, N, cells, seed=2, radius=0.45)
    res = []
    for cls in (pyoracle.LimitingMesh, pyoracle.RefLimitingMesh):
        m = cls(dim, N, cells, (1.0,) * dim, bc)
        m.set_solution(u)
        m.set_fv_initial(fv)
        m.init(0.0)
        masks = []
        for _ in range(steps):
            m.step(1)
            masks.append(m.status().copy())
        res.append((m.get_solution(), np.array(masks), m.state()))
    (a, ma, sa), (b, mb, sb) = res
    assert np.array_equal(ma, mb)
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-13
    assert sa["irregular_steps"] == sb["irregular_steps"]
    # FV-active cells on the domain boundary
    st = ma.reshape(steps, *reversed(cells))
    edge = np.zeros(st.shape[1:], bool)
    for ax in range(dim):
        idx = [slice(None)] * dim
        idx[ax] = 0
        edge[tuple(idx)] = True
        idx[ax] = -1
        edge[tuple(idx)] = True
    assert (st[:, edge] >= 2).any()


def test_reflective_dg_mesh_vs_reference():
    """a pressure pulse at rest between reflective walls (DG only)"""
    cells = (9, 9)
    u, _ = problems.gaussian_pulse_2d(3, cells, seed=10)
    u[..., 1:4] = 0.0
    u[..., 4] = u[..., 0] / 0.4
    res = []
    for impl in ("oracle", "ref"):
        m = pyoracle.Mesh(2, 3, cells, [1.0, 1.0], 1, impl=impl, nthreads=4)
        m.set_solution(u)
        m.init(0.0)
        m.step(15)
        res.append((m.get_solution(), m.state()))
    (a, sa), (b, sb) = res
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-13
    assert sa["picard_sweeps"] == sb["picard_sweeps"]
