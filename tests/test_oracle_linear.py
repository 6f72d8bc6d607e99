"""The C oracle's linear kernels (oracle/linear.c) pinned against the
reference's own kernel-test vectors and against the reference's linear
kernels compiled from source (oracle/_ref):

* generic Euler mock (GenericEulerKernelTest{2D,3D}.cpp): volumeIntegralLinear,
  surfaceIntegralLinear, riemannSolverLinear; absolute tolerance 1e-10
  (GenericEulerKernelTest.h:69);
* elastic waves (ElasticityKernelTest2D.cpp, N = 4, 9 variables, 3
  parameters): riemannSolverLinear, volumeIntegralLinear,
  surfaceIntegralLinear and spaceTimePredictorLinear (that test is switched
  off in the reference's run(), its data still match the reference kernels
  and this oracle), tolerance 1e-9 (ElasticityKernelTest.h:61).
"""
import numpy as np
import pytest

import pyoracle
from exahype_b200 import problems

EPS = 1e-10


def widen(a, nvar, ndata):
    a = np.asarray(a).reshape(-1, nvar)
    out = np.zeros((a.shape[0], ndata))
    out[:, :nvar] = a
    return out


def test_volume_integral_linear_golden(golden):
    # GenericEulerKernelTest2D.cpp:692-745, GenericEulerKernelTest3D.cpp:162-194
    k2 = pyoracle.Kernels(2, 3, pde=1)
    g = "2d/generic_euler/"
    du = k2.lin_volume_integral(golden[g + "testVolumeIntegral/lFhi"][:160], [3.70370370370370349811e-02] * 2)
    np.testing.assert_allclose(du, golden[g + "testVolumeIntegralLinear/lduh_1"], rtol=0, atol=EPS)
    lf = np.zeros(160)
    lf[1:80:5] = 1.0
    lf[80 + 2::5] = 1.0
    du = k2.lin_volume_integral(lf, [0.05] * 2)
    np.testing.assert_allclose(du, golden[g + "testVolumeIntegralLinear/lduh_2"], rtol=0, atol=EPS)
    k3 = pyoracle.Kernels(3, 3, pde=1)
    lf = np.zeros(960)
    lf[1:320:5] = 1.0
    lf[320 + 2:640:5] = 2.0
    lf[640 + 3::5] = 3.0
    du = k3.lin_volume_integral(lf, [0.5] * 3)
    np.testing.assert_allclose(du, golden["3d/generic_euler/testVolumeIntegralLinear/lduh"], rtol=0, atol=EPS)


def test_surface_integral_linear_golden(golden):
    # GenericEulerKernelTest2D.cpp:191-262, GenericEulerKernelTest3D.cpp:230-272
    k2 = pyoracle.Kernels(2, 3, pde=1)
    g = "2d/generic_euler/"
    fb = np.zeros(80)
    fb[0 + 1:20:5] = fb[20 + 1:40:5] = 1.0
    fb[40 + 2:60:5] = fb[60 + 2:80:5] = 1.0
    du = k2.lin_surface_integral(golden[g + "testSurfaceIntegral/lduh_in"], fb, [0.1] * 2)
    np.testing.assert_allclose(du, golden[g + "testSurfaceIntegralLinear/lduh_out_1"], rtol=0, atol=EPS)
    du = k2.lin_surface_integral(golden[g + "testSurfaceIntegral/lduh_in"], golden[g + "testSurfaceIntegral/lFhbnd_in"],
                                 [0.1] * 2)
    np.testing.assert_allclose(du, golden[g + "testSurfaceIntegralLinear/lduh_out_2"], rtol=0, atol=EPS)
    k3 = pyoracle.Kernels(3, 3, pde=1)
    fb = np.zeros(480)
    for f, v in ((0, 1), (1, 1), (2, 2), (3, 2), (4, 3), (5, 3)):
        fb[f * 80 + v:(f + 1) * 80:5] = 1.0
    du = k3.lin_surface_integral(np.arange(320) / 10.0, fb, [0.1] * 3)
    np.testing.assert_allclose(du, golden["3d/generic_euler/testSurfaceIntegralLinear/lduh"], rtol=0, atol=EPS)


def test_riemann_linear_golden(golden):
    # GenericEulerKernelTest2D.cpp:344-460 (normals 0 and 1), GenericEulerKernelTest3D.cpp:324-400 (normal 1):
    # the mock's system matrix is zero, so the fluctuations are the scalar dissipation alone
    k2 = pyoracle.Kernels(2, 3, pde=1)
    g = "2d/generic_euler/"
    QL, QR = widen(golden[g + "testRiemannSolver/QL"], 5, 6), widen(golden[g + "testRiemannSolver/QR"], 5, 6)
    for normal, sfx in ((0, "1"), (1, "2")):
        FL, FR = k2.lin_riemann(QL, QR, normal)
        np.testing.assert_allclose(FL, golden[g + "testRiemannSolverLinear/FL_" + sfx], rtol=0, atol=EPS)
        np.testing.assert_allclose(FR, golden[g + "testRiemannSolverLinear/FR_" + sfx], rtol=0, atol=EPS)
    k3 = pyoracle.Kernels(3, 3, pde=1)
    g = "3d/generic_euler/"
    QL, QR = widen(golden[g + "testRiemannSolver/QL"], 5, 6), widen(golden[g + "testRiemannSolver/QR"], 5, 6)
    FL, FR = k3.lin_riemann(QL, QR, 1)
    np.testing.assert_allclose(FL, golden[g + "testRiemannSolverLinear/FL"], rtol=0, atol=EPS)
    np.testing.assert_allclose(FR, golden[g + "testRiemannSolverLinear/FR"], rtol=0, atol=EPS)


ELASTIC_DX = [38.4615384615385, 35.7142857142857]  # ElasticityKernelTest2D.cpp


def elastic_state(golden, var, par, n):
    g = "2d/elasticity/"
    return np.concatenate([golden[g + var].reshape(n, 9), golden[g + par].reshape(n, 3)], axis=1)


def test_elastic_kernels_golden(golden):
    # ElasticityKernelTest2D.cpp:237-303 (Riemann, normal 1), :306-410 (predictor),
    # :440-487 (volume integral), :489-528 (surface integral)
    k = pyoracle.Kernels(2, 4, pde=2)
    g = "2d/elasticity/"
    qL = elastic_state(golden, "testRiemannSolverLinear/qL_IN", "testRiemannSolverLinear/paramL_IN", 5)
    qR = elastic_state(golden, "testRiemannSolverLinear/qR_IN", "testRiemannSolverLinear/paramR_IN", 5)
    FL, FR = k.lin_riemann(qL, qR, 1)
    np.testing.assert_allclose(FL, golden[g + "testRiemannSolverLinear/FL_OUT"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(FR, golden[g + "testRiemannSolverLinear/FR_OUT"], rtol=0, atol=1e-9)
    du = k.lin_volume_integral(golden[g + "testVolumeIntegralLinear/lFhi_IN"], ELASTIC_DX)
    np.testing.assert_allclose(du, golden[g + "testVolumeIntegralLinear/lduh_OUT"], rtol=0, atol=1e-9)
    du = k.lin_surface_integral(golden[g + "testSurfaceIntegralLinear/lduh_IN"],
                                golden[g + "testSurfaceIntegralLinear/lFbnd_IN"], ELASTIC_DX)
    np.testing.assert_allclose(du, golden[g + "testSurfaceIntegralLinear/lduh_OUT"], rtol=0, atol=1e-9)
    luh = elastic_state(golden, "testSpaceTimePredictorLinear/luh_IN", "testSpaceTimePredictorLinear/param_IN", 25)
    out = k.lin_predictor(luh, ELASTIC_DX, 0.813172798364530)
    p = g + "testSpaceTimePredictorLinear/"
    np.testing.assert_allclose(out["lQhi"].reshape(25, 12)[:, :9].ravel(), golden[p + "lQhi_OUT"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(out["lFhi"], golden[p + "lFhi_OUT"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(out["lQhbnd"].reshape(20, 12)[:, :9].ravel(), golden[p + "lQbnd_OUT"], rtol=0,
                               atol=1e-9)
    np.testing.assert_allclose(out["lFhbnd"], golden[p + "lFbnd_OUT"], rtol=0, atol=1e-9)


def random_elastic(rng, n):
    return np.concatenate([rng.normal(size=(n, 9)), rng.uniform(1, 3, size=(n, 1)), rng.uniform(0.5, 1.5, size=(n, 1)),
                           rng.uniform(1, 2, size=(n, 1))], axis=1)


needs_ref = pytest.mark.skipif(not (pyoracle.ref_available(2) and pyoracle.ref_available(3)),
                               reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("dim,N", [(2, 3), (2, 4), (2, 5), (3, 3), (3, 4), (3, 5)])
def test_elastic_kernels_vs_reference(dim, N):
    """oracle vs the reference's linear kernels compiled from source; the two
    differ only through the operator tables (the oracle's generated tables
    equal the reference's to 1e-15), the time step is bit-identical"""
    rng = np.random.default_rng(dim * 10 + N)
    o, r = pyoracle.Kernels(dim, N, 2), pyoracle.Kernels(dim, N, 2, impl="ref")
    P, F = (N + 1) ** dim, (N + 1) ** (dim - 1)
    u = random_elastic(rng, P)
    dx = [0.1, 0.12, 0.09][:dim]
    a, b = o.lin_predictor(u, dx, 3e-3), r.lin_predictor(u, dx, 3e-3)
    for key in a:
        assert np.max(np.abs(a[key] - b[key])) <= 1e-13 * max(np.max(np.abs(b[key])), 1.0), key
    QL, QR = random_elastic(rng, F), random_elastic(rng, F)
    for d in range(dim):
        (x1, x2), (y1, y2) = o.lin_riemann(QL, QR, d), r.lin_riemann(QL, QR, d)
        assert np.max(np.abs(x1 - y1)) <= 1e-13 * np.max(np.abs(y1)) and np.max(np.abs(x2 - y2)) <= 1e-13 * np.max(np.abs(y2))
    fb, du = rng.normal(size=2 * dim * F * 9), rng.normal(size=P * 9)
    x, y = o.lin_surface_integral(du, fb, dx), r.lin_surface_integral(du, fb, dx)
    assert np.max(np.abs(x - y)) <= 1e-13 * np.max(np.abs(y))
    assert o.stable_dt(u, dx) == r.stable_dt(u, dx)


@needs_ref
@pytest.mark.parametrize("dim,N,cells,steps", [(2, 4, (8, 8), 10), (3, 3, (4, 4, 4), 4)])
def test_elastic_mesh_vs_reference(dim, N, cells, steps):
    """uniform periodic mesh, linear scheme: the oracle harness over the C
    restatement vs over the reference's linear kernels"""
    u, _ = problems.elastic_pulse(dim, N, cells, seed=5)
    res = []
    for impl in ("oracle", "ref"):
        m = pyoracle.Mesh(dim, N, cells, [1.0] * dim, -1, pde=2, impl=impl, nthreads=4)
        m.set_solution(u)
        m.init(0.0)
        m.step(steps)
        res.append((m.get_solution(), m.state()))
    (a, sa), (b, sb) = res
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-13
    assert sa["dt"] == sb["dt"] and sa["steps"] == sb["steps"] == steps
    # parameters are carried unchanged
    assert np.array_equal(a[..., 9:], u[..., 9:])


@needs_ref
@pytest.mark.parametrize("dim,N", [(2, 3), (2, 5), (3, 3), (3, 5)])
def test_elastic_boundary_faces_vs_reference(dim, N):
    """boundaryConditions + riemannSolverLinear on every face of a cell, for
    outflow (the inside state copied: no jump, no fluctuation) and a rigid
    wall (velocities negated)"""
    rng = np.random.default_rng(7 * dim + N)
    o, r = pyoracle.Kernels(dim, N, 2), pyoracle.Kernels(dim, N, 2, impl="ref")
    F = (N + 1) ** (dim - 1)
    QIn = random_elastic(rng, F)
    FIn = rng.normal(size=F * 9)
    for face in range(2 * dim):
        for kind in (0, 1):
            a = o.lin_boundary_face(FIn, QIn, face, kind)
            b = r.lin_boundary_face(FIn, QIn, face, kind)
            assert np.max(np.abs(a - b)) <= 1e-14 * max(np.max(np.abs(b)), 1.0), (face, kind)
            if kind == 0:
                assert np.max(np.abs(a)) == 0.0
            else:
                assert np.max(np.abs(a)) > 0.1
    # a wall against a state at rest leaves stresses only: the fluctuation is
    # that of the velocity jump alone, so a zero-velocity state gives zero
    Q0 = QIn.copy()
    Q0[:, 6:9] = 0.0
    assert np.max(np.abs(o.lin_boundary_face(FIn, Q0, 0, 1))) == 0.0


@needs_ref
@pytest.mark.parametrize("dim,N,cells,bc,steps", [(2, 4, (8, 8), 0, 8), (2, 3, (8, 6), [1, 1, 0, 1], 8),
                                                  (3, 3, (4, 4, 4), 1, 3)])
def test_elastic_mesh_boundaries_vs_reference(dim, N, cells, bc, steps):
    """uniform elastic meshes with outflow and rigid-wall domain faces: the
    oracle harness over the C restatement vs over the reference's kernels"""
    u, _ = problems.elastic_pulse(dim, N, cells, seed=9)
    res = []
    for impl in ("oracle", "ref"):
        m = pyoracle.Mesh(dim, N, cells, [1.0] * dim, bc, pde=2, impl=impl, nthreads=4)
        m.set_solution(u)
        m.init(0.0)
        m.step(steps)
        res.append((m.get_solution(), m.state()))
    (a, sa), (b, sb) = res
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-13
    assert sa["dt"] == sb["dt"] and sa["steps"] == sb["steps"] == steps
    # the boundaries change the solution against the periodic mesh
    m = pyoracle.Mesh(dim, N, cells, [1.0] * dim, -1, pde=2, nthreads=4)
    m.set_solution(u)
    m.init(0.0)
    m.step(steps)
    assert np.linalg.norm(m.get_solution() - a) / np.linalg.norm(a) > 1e-8
