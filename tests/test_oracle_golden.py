"""Pins the C oracle against the reference's own kernel-test vectors
(ExaHyPE/exahype/tests/kernels/c/GenericEulerKernelTest{2D,3D}.cpp), with the
reference tests' absolute tolerance eps = 1e-10 (GenericEulerKernelTest.h:69).
The mock PDE there is the "2.5D" Euler with one material parameter (pde=1)."""
import numpy as np
import pytest

import pyoracle

EPS = 1e-10


def widen(a, nvar, ndata):
    """test data is nVar-strided; the kernels see nData = nVar + nPar."""
    a = a.reshape(-1, nvar)
    out = np.zeros((a.shape[0], ndata))
    out[:, :nvar] = a
    return out


@pytest.mark.parametrize("dim,dt", [(2, 1.686854344081342e-3), (3, 1.083937460199773e-3)])
def test_predictor_golden(golden, dim, dt):
    # GenericEulerKernelTest2D.cpp:895-1035, GenericEulerKernelTest3D.cpp:611-~760
    k = pyoracle.Kernels(dim, 3, pde=1)
    g = "%dd/generic_euler/testSpaceTimePredictorNonlinear/" % dim
    luh = widen(golden[g + "luh"], 5, 6)
    out = k.predictor(luh, [0.05] * dim, dt, temps=True)
    b, nV, nD = 4, 5, 6
    lQi = out["lQi"].reshape(-1, nD)[:, :nV].ravel()
    np.testing.assert_allclose(lQi, golden[g + "lQi"], rtol=0, atol=EPS)
    # lFi: reference stores (t,z,y,x,dim+1,var); golden (t,z,y,x,dim,var)
    lFi = out["lFi"].reshape(-1, dim + 1, nV)[:, :dim, :].ravel()
    np.testing.assert_allclose(lFi, golden[g + "lFi"], rtol=0, atol=EPS)
    lQhi = out["lQhi"].reshape(-1, nD)[:, :nV].ravel()
    np.testing.assert_allclose(lQhi, golden[g + "lQhi"], rtol=0, atol=EPS)
    nflux = dim * nV * b ** dim
    np.testing.assert_allclose(out["lFhi"][:nflux], golden[g + "lFhi"][:nflux], rtol=0, atol=EPS)
    lQhbnd = out["lQhbnd"].reshape(-1, nD)[:, :nV].ravel()
    np.testing.assert_allclose(lQhbnd, golden[g + "lQhbnd"], rtol=0, atol=EPS)
    np.testing.assert_allclose(out["lFhbnd"], golden[g + "lFhbnd"], rtol=0, atol=EPS)
    assert 1 <= out["iterations"] <= 8


def test_riemann_golden_2d(golden):
    # GenericEulerKernelTest2D.cpp:499-690, tests 1-3
    k = pyoracle.Kernels(2, 3, pde=1)
    g = "2d/generic_euler/testRiemannSolverNonlinear/"
    # test 1: constant state -> FL == FR
    Q = widen(np.tile([1., 0., 0., 0., 2.5], 4), 5, 6)
    FL, FR = k.riemann(np.zeros(20), np.zeros(20), Q, Q, 0)
    assert np.array_equal(FL, FR)
    for t, d in (("1", 0), ("2", 1)):
        QL = widen(golden[g + "QL_%s_in" % t], 5, 6)
        QR = widen(golden[g + "QR_%s_in" % t], 5, 6)
        FL, FR = k.riemann(golden[g + "FL_%s_in" % t], golden[g + "FR_%s_in" % t], QL, QR, d)
        np.testing.assert_allclose(FL, golden[g + "F_%s_out" % t], rtol=0, atol=EPS)
        np.testing.assert_allclose(FR, golden[g + "F_%s_out" % t], rtol=0, atol=EPS)


def test_riemann_golden_3d(golden):
    # GenericEulerKernelTest3D.cpp:408-489
    k = pyoracle.Kernels(3, 3, pde=1)
    n = 5 * 16
    FL = np.arange(n, dtype=np.float64) + 1
    FR = np.arange(n, dtype=np.float64) - 1
    QL = widen(golden["3d/generic_euler/testRiemannSolver/QL"], 5, 6)
    QR = widen(golden["3d/generic_euler/testRiemannSolver/QR"], 5, 6)
    FL, FR = k.riemann(FL, FR, QL, QR, 1)
    np.testing.assert_allclose(FL, golden["3d/generic_euler/testRiemannSolverNonlinear/FL"], rtol=0, atol=EPS)
    np.testing.assert_allclose(FR, golden["3d/generic_euler/testRiemannSolverNonlinear/FR"], rtol=0, atol=EPS)


def test_surface_integral_golden_2d(golden):
    # GenericEulerKernelTest2D.cpp:265-342
    k = pyoracle.Kernels(2, 3, pde=1)
    lduh_in = golden["2d/generic_euler/testSurfaceIntegral/lduh_in"]
    lF = np.zeros(80)
    for i in range(0, 20, 5):
        lF[i + 1] = 1.0
        lF[20 + i + 1] = 1.0
        lF[40 + i + 2] = 1.0
        lF[60 + i + 2] = 1.0
    out = k.surface_integral(lduh_in, lF, [0.1, 0.1])
    np.testing.assert_allclose(out, golden["2d/generic_euler/testSurfaceIntegralNonlinear/lduh_1"], rtol=0, atol=EPS)
    out = k.surface_integral(lduh_in, golden["2d/generic_euler/testSurfaceIntegral/lFhbnd_in"], [0.1, 0.1])
    np.testing.assert_allclose(out, golden["2d/generic_euler/testSurfaceIntegralNonlinear/lduh_2"], rtol=0, atol=EPS)


def test_solution_update_golden_3d(golden):
    # GenericEulerKernelTest3D.cpp:491-528 (the test compares the first b^2 nodes)
    k = pyoracle.Kernels(3, 3, pde=1)
    luh = np.zeros((64, 6))
    luh[:, 0] = 1.0
    luh[:, 4] = 2.5
    lduh = np.arange(5 * 64, dtype=np.float64)
    out = k.solution_update(luh, lduh, 1.40831757919882352703e-03).reshape(64, 6)[:, :5].ravel()
    np.testing.assert_allclose(out[:80], golden["3d/generic_euler/testSolutionUpdate/luh"][:80], rtol=0, atol=EPS)


def test_pde_fluxes_golden(golden):
    # GenericEulerKernelTest{2D,3D}.cpp: testPDEFluxes, Q = {1, .1, .2, .3, 3.5}
    for dim in (2, 3):
        s = pyoracle._Solver(dim, 3, 1)
        Q = np.array([1.0, 0.1, 0.2, 0.3, 3.5, 0.0])
        F = np.zeros(3 * 5)
        pyoracle.lib().orc_flux(pyoracle.ctypes.byref(s), pyoracle._p(Q), pyoracle._p(F))
        for d, name in enumerate("fgh"[:dim]):
            np.testing.assert_allclose(F[5 * d:5 * d + 5], golden["%dd/generic_euler/testPDEFluxes/%s" % (dim, name)],
                                       rtol=0, atol=EPS)


@pytest.mark.parametrize("dim", [2, 3])
def test_limiter_projections_golden(golden, dim):
    """limiter_testdata.cpp (LimiterKernelTest, N = 3, nVar = 5, no ghost
    layers): luh -> subcell averages, luh -> Lobatto values, subcells -> luh."""
    import ctypes
    N, b, B, E, nV = 3, 4, 7, 11, 5
    s = pyoracle._Solver(dim, N, 0)
    g = "%dd/limiter/" % dim
    luh = np.ascontiguousarray(golden[g + "testFromLuhConversion/luh_in"])
    lim = np.zeros((E,) * dim + (nV,))
    pyoracle.lib().orc_project_fv(ctypes.byref(s), pyoracle._p(luh), pyoracle._p(lim.reshape(-1)))
    inner = lim[(slice(2, -2),) * dim].reshape(-1)
    np.testing.assert_allclose(inner, golden[g + "testFromLuhConversion/lim_out"], rtol=0, atol=1e-10)
    # Lobatto values with the generated uh2lob table ([j][i]: basis j at node i)
    L = pyoracle.table("uh2lob", N).reshape(b, b)
    u = luh.reshape((b,) * dim + (nV,))
    lob = np.einsum("yxv,ya,xb->abv", u, L, L) if dim == 2 else np.einsum("zyxv,zc,ya,xb->cabv", u, L, L, L)
    np.testing.assert_allclose(lob.reshape(-1), golden[g + "testFromLuhConversion/lob_out"], rtol=0, atol=1e-10)
    lim2 = np.zeros((E,) * dim + (nV,))
    lim2[(slice(2, -2),) * dim] = golden[g + "testToLuhConversion/lim_in"].reshape((B,) * dim + (nV,))
    out = np.zeros(b ** dim * nV)
    pyoracle.lib().orc_project_dg(ctypes.byref(s), pyoracle._p(np.ascontiguousarray(lim2.reshape(-1))),
                                  pyoracle._p(out))
    np.testing.assert_allclose(out, golden[g + "testToLuhConversion/luh_out"], rtol=0, atol=1e-10)

