"""The oracle's source / non-conservative-product paths (pde 3: the kernel
tests' Euler mock with an algebraic source and the tests' non-zero product
mock) against the reference's own templates instantiated with
useSource = useNCP = true and compiled from its sources (oracle/_ref):
spaceTimePredictorNonlinear with its temporaries, volumeIntegralNonlinear
<useSourceOrNCP>, riemannSolverNonlinear<useNCP> on interior and boundary
faces, and uniform-mesh runs. CPU only."""
import numpy as np
import pytest

import pyoracle

pytestmark = pytest.mark.skipif(not pyoracle.ref_available(2), reason="oracle/_ref not built")


def states(rng, n, ndata=6):
    u = np.zeros((n, ndata))
    u[:, 0] = 1.0 + 0.2 * rng.random(n)
    u[:, 1:4] = 0.2 * (rng.random((n, 3)) - 0.5)
    u[:, 4] = 2.5 + 0.3 * rng.random(n)
    u[:, 5] = rng.random(n)
    return u


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("dim,order", [(2, 3), (2, 5), (3, 3), (3, 5)])
def test_predictor_and_volume_integral(dim, order):
    rng = np.random.default_rng(dim * 10 + order)
    P = (order + 1) ** dim
    luh = states(rng, P)
    dx = [0.05, 0.04, 0.045][:dim]
    o = pyoracle.Kernels(dim, order, pde=3).predictor(luh, dx, 1e-3, temps=True)
    r = pyoracle.Kernels(dim, order, pde=3, impl="ref").predictor(luh, dx, 1e-3, temps=True)
    assert o["iterations"] == r["iterations"]
    for key in ("lQi", "lFi", "lQhi", "lFhi", "lQhbnd", "lFhbnd", "lduh"):
        assert rel(o[key], r[key]) < 1e-13, key
    # the source block of lFi / lFhi is non-zero, and so is what it adds to lduh
    nV = 5
    lFhi = o["lFhi"].reshape(dim + 1, P, nV)
    assert np.abs(lFhi[dim]).max() > 0.1
    plain = pyoracle.Kernels(dim, order, pde=1).predictor(luh, dx, 1e-3)
    assert rel(o["lduh"], plain["lduh"]) > 1e-3


@pytest.mark.parametrize("dim,order", [(2, 3), (3, 5)])
def test_riemann_fluctuations(dim, order):
    rng = np.random.default_rng(5 + dim)
    F = (order + 1) ** (dim - 1)
    QL, QR = states(rng, F), states(rng, F)
    FL0, FR0 = rng.standard_normal((F, 5)), rng.standard_normal((F, 5))
    ko = pyoracle.Kernels(dim, order, pde=3)
    kr = pyoracle.Kernels(dim, order, pde=3, impl="ref")
    for d in range(dim):
        a = ko.riemann(FL0.copy(), FR0.copy(), QL, QR, d)
        b = kr.riemann(FL0.copy(), FR0.copy(), QL, QR, d)
        assert rel(a[0], b[0]) < 1e-14 and rel(a[1], b[1]) < 1e-14
        assert np.abs(a[0] - a[1]).max() > 0.1  # the product splits the two sides
    for f in range(2 * dim):
        a = ko.boundary_face(FL0.copy(), QL, f)
        b = kr.boundary_face(FL0.copy(), QL, f)
        assert rel(a, b) < 1e-14


@pytest.mark.parametrize("dim,order,cells,steps", [(2, 3, (8, 8), 4), (3, 3, (4, 4, 4), 2)])
def test_mesh_runs(dim, order, cells, steps):
    from exahype_b200 import problems
    if dim == 2:
        u, _ = problems.gaussian_pulse_2d(order, cells, seed=3)
    else:
        u, _ = problems.gaussian_pulses_3d(order, cells, seed=3)
    u6 = np.concatenate([u, np.zeros(u.shape[:-1] + (1,))], axis=-1)
    runs = []
    for impl in ("oracle", "ref"):
        m = pyoracle.Mesh(dim, order, cells, [1.0] * dim, -1, pde=3, impl=impl, nthreads=4)
        m.set_solution(u6)
        m.init(0.0)
        m.step(steps)
        runs.append((m.get_solution(), m.state()))
    (a, sa), (b, sb) = runs
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    assert sa["picard_sweeps"] == sb["picard_sweeps"] and sa["steps"] == sb["steps"] == steps
    # the source and the product change the solution against the plain mock
    m = pyoracle.Mesh(dim, order, cells, [1.0] * dim, -1, pde=1, nthreads=4)
    m.set_solution(u6)
    m.init(0.0)
    m.step(steps)
    assert np.linalg.norm(m.get_solution() - a) / np.linalg.norm(a) > 1e-4
