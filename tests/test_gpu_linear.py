"""GPU parity of the linear ADER-DG kernels (Cauchy-Kovalevski predictor,
linear Riemann solver, linear volume and surface integrals) with the elastic
wave PDE, through the C ABI.

Bars: the reference's elasticity kernel-test vectors replayed on the GPU with
their tolerance 1e-9 (ElasticityKernelTest.h:61); against the C oracle 1e-12
relative (max-norm per array, relative L2 for mesh runs); time-step sizes
bit-identical; step counts equal.
"""
import numpy as np
import pytest

import pyoracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

RTOL = 1e-12
ELASTIC_DX = [38.4615384615385, 35.7142857142857]  # ElasticityKernelTest2D.cpp


@pytest.fixture(scope="module")
def eb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import exahype_b200
    exahype_b200.load()
    return exahype_b200


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def zeros(n):
    return torch.zeros(int(n), device="cuda", dtype=torch.float64)


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def random_elastic(rng, n, P):
    u = np.zeros((n, P, 12))
    u[..., :9] = rng.normal(size=(n, P, 9))
    u[..., 9] = rng.uniform(1, 3, size=(n, P))
    u[..., 10] = rng.uniform(0.5, 1.5, size=(n, P))
    u[..., 11] = rng.uniform(1, 2, size=(n, P))
    return u


def elastic_state(golden, var, par, n):
    g = "2d/elasticity/"
    return np.concatenate([golden[g + var].reshape(n, 9), golden[g + par].reshape(n, 3)], axis=1)


@pytest.mark.parametrize("variant", [0, 1])
def test_predictor_linear_golden_gpu(eb, golden, variant):
    """ElasticityKernelTest2D::testSpaceTimePredictorLinear (N = 4) replayed on
    the GPU: time averages and boundary extrapolations"""
    s = eb.Solver(2, 4, eb.PDE_ELASTIC)
    s.variant = variant
    p = "2d/elasticity/testSpaceTimePredictorLinear/"
    luh = dev(elastic_state(golden, "testSpaceTimePredictorLinear/luh_IN", "testSpaceTimePredictorLinear/param_IN", 25))
    qb, fb, du, qh, fh = zeros(4 * 5 * 12), zeros(4 * 5 * 9), zeros(25 * 9), zeros(25 * 12), zeros(2 * 25 * 9)
    s.space_time_predictor_linear_temps(luh, qb, fb, du, dev([0.813172798364530]), ELASTIC_DX, 1, qh, fh)
    np.testing.assert_allclose(host(qh).reshape(25, 12)[:, :9].ravel(), golden[p + "lQhi_OUT"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(host(fh), golden[p + "lFhi_OUT"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(host(qb).reshape(20, 12)[:, :9].ravel(), golden[p + "lQbnd_OUT"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(host(fb), golden[p + "lFbnd_OUT"], rtol=0, atol=1e-9)
    # the parameters' extrapolations and the volume integral against the oracle
    r = pyoracle.Kernels(2, 4, pde=2).lin_predictor(host(luh), ELASTIC_DX, 0.813172798364530)
    assert rel(host(qb), r["lQhbnd"]) < RTOL and rel(host(du), r["lduh"]) < RTOL


def test_riemann_and_volume_linear_golden_gpu(eb, golden):
    """ElasticityKernelTest2D::testRiemannSolverLinear (normal 1) and
    ::testVolumeIntegralLinear replayed on the GPU"""
    s = eb.Solver(2, 4, eb.PDE_ELASTIC)
    g = "2d/elasticity/"
    qL = elastic_state(golden, "testRiemannSolverLinear/qL_IN", "testRiemannSolverLinear/paramL_IN", 5)
    qR = elastic_state(golden, "testRiemannSolverLinear/qR_IN", "testRiemannSolverLinear/paramR_IN", 5)
    # two cells: cell 0's face 3 (+y) meets cell 1's face 2 (-y)
    qb = np.zeros((2, 4, 5, 12))
    qb[0, 3], qb[1, 2] = qL, qR
    qbd, fbd = dev(qb), zeros(2 * 4 * 5 * 9)
    ints = lambda a: dev(np.array(a, dtype=np.int32), torch.int32)
    s.riemann_solver_linear(qbd, fbd, ints([0]), ints([1]), ints([1]), 1)
    fb = host(fbd).reshape(2, 4, 5 * 9)
    np.testing.assert_allclose(fb[0, 3], golden[g + "testRiemannSolverLinear/FL_OUT"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(fb[1, 2], golden[g + "testRiemannSolverLinear/FR_OUT"], rtol=0, atol=1e-9)
    du = zeros(25 * 9)
    s.volume_integral_linear(du, dev(golden[g + "testVolumeIntegralLinear/lFhi_IN"]), 1)
    np.testing.assert_allclose(host(du), golden[g + "testVolumeIntegralLinear/lduh_OUT"], rtol=0, atol=1e-9)


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("dim,N", [(2, 3), (2, 4), (2, 5), (3, 3), (3, 4), (3, 5)])
def test_linear_kernels_vs_oracle(eb, dim, N, variant):
    """predictor + volume integral, Riemann solver and corrector (linear
    surface integral, update, admissible step) on random elastic cells"""
    rng = np.random.default_rng(100 * dim + N)
    s = eb.Solver(dim, N, eb.PDE_ELASTIC)
    s.variant = variant
    o = pyoracle.Kernels(dim, N, pde=2)
    b = N + 1
    P, F, n = b ** dim, b ** (dim - 1), 37
    u = random_elastic(rng, n, P)
    dx, dt = [0.1, 0.12, 0.09][:dim], 3e-3
    qb, fb, du = zeros(n * 2 * dim * F * 12), zeros(n * 2 * dim * F * 9), zeros(n * P * 9)
    s.space_time_predictor_linear(dev(u), qb, fb, du, dev([dt]), dx, n)
    qb_h, fb_h, du_h = host(qb).reshape(n, -1), host(fb).reshape(n, -1), host(du).reshape(n, -1)
    for c in range(n):
        r = o.lin_predictor(u[c], dx, dt)
        assert rel(qb_h[c], r["lQhbnd"]) < RTOL and rel(fb_h[c], r["lFhbnd"]) < RTOL and rel(du_h[c], r["lduh"]) < RTOL
    # Riemann: faces between consecutive cells in direction c % dim
    nf = n - 1
    fl, fr, fd = np.arange(nf, dtype=np.int32), np.arange(1, n, dtype=np.int32), (np.arange(nf) % dim).astype(np.int32)
    qb_r = rng.normal(size=(n, 2 * dim, F, 12))
    qb_r[..., 9] = rng.uniform(1, 3, size=qb_r.shape[:-1])
    qb_r[..., 10] = rng.uniform(0.5, 1.5, size=qb_r.shape[:-1])
    qb_r[..., 11] = rng.uniform(1, 2, size=qb_r.shape[:-1])
    fbd = zeros(n * 2 * dim * F * 9)
    ints = lambda a: dev(a, torch.int32)
    s.riemann_solver_linear(dev(qb_r), fbd, ints(fl), ints(fr), ints(fd), nf)
    got = host(fbd).reshape(n, 2 * dim, F * 9)
    for f in range(nf):
        d = fd[f]
        FL, FR = o.lin_riemann(qb_r[fl[f], 2 * d + 1], qb_r[fr[f], 2 * d], d)
        assert rel(got[fl[f], 2 * d + 1], FL) < RTOL and rel(got[fr[f], 2 * d], FR) < RTOL
    # corrector: linear surface integral + update + admissible step
    lduh = rng.normal(size=(n, P * 9))
    lfb = rng.normal(size=(n, 2 * dim * F * 9))
    luh = dev(u)
    dtmin = dev([0.0])
    eb.Solver.reset_min(dtmin)
    s.corrector(luh, dev(lduh), dev(lfb), dev([dt]), dtmin, dx, n)
    got = host(luh).reshape(n, -1)
    want_dt = np.inf
    for c in range(n):
        d_ = o.lin_surface_integral(lduh[c], lfb[c], dx)
        un = o.solution_update(u[c].ravel(), d_, dt)
        assert rel(got[c], un) < RTOL
        want_dt = min(want_dt, o.stable_dt(un, dx))
    assert host(dtmin)[0] == want_dt  # bit-identical admissible step


@pytest.mark.parametrize("dim,N,cells,steps", [(2, 4, (16, 16), 20), (2, 3, (12, 12), 15), (3, 3, (6, 6, 6), 10),
                                               (3, 5, (4, 4, 4), 6)])
def test_elastic_mesh_vs_oracle(eb, dim, N, cells, steps):
    from exahype_b200 import problems
    u, _ = problems.elastic_pulse(dim, N, cells, seed=11)
    s = eb.Solver(dim, N, eb.PDE_ELASTIC)
    m = eb.Mesh(s, cells, [0.0] * dim, [1.0] * dim, eb.BC_PERIODIC)
    m.set_solution(u)
    m.init(0.0)
    m.step(steps)
    o = pyoracle.Mesh(dim, N, cells, [1.0] * dim, -1, pde=2, nthreads=8)
    o.set_solution(u)
    o.init(0.0)
    o.step(steps)
    a, b = m.get_solution(), o.get_solution()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < RTOL
    assert np.array_equal(a[..., 9:], u[..., 9:])
    sa, sb = m.state(), o.state()
    assert sa["steps"] == sb["steps"] == steps and sa["dt"] == sb["dt"] and sa["t"] == sb["t"]
    n_g, n_o = m.run_until(sa["t"] + 5.5 * sa["dt"]), o.run_until(sb["t"] + 5.5 * sb["dt"])
    assert n_g == n_o == 6


def test_linear_solver_api_errors(eb):
    s = eb.Solver(2, 4, eb.PDE_ELASTIC)
    assert s.nvar == 9 and s.ndata == 12 and s.linear
    x = zeros(4)
    with pytest.raises(eb.ExaError):
        s.space_time_predictor(x, x, x, x, x, [1, 1], 1)  # the nonlinear predictor rejects a linear solver
    with pytest.raises(eb.ExaError):
        eb.Mesh(s, (4, 4), [0, 0], [1, 1], [eb.BC_OUTFLOW, eb.BC_PERIODIC, 0, 0])  # periodic on one face only
    e = eb.Solver(2, 3, eb.PDE_EULER)
    with pytest.raises(eb.ExaError):
        e.riemann_solver_linear(x, x, None, None, None, 0)  # and the linear kernels reject a nonlinear one
    chosen, ms = s.autotune(64)
    assert chosen in (0, 1) and ms[0] > 0 and ms[1] > 0 and all(v == -1.0 for v in ms[2:])


@pytest.mark.parametrize("dim,N", [(2, 3), (2, 5), (3, 3), (3, 5)])
def test_linear_boundary_faces_vs_oracle_and_reference(eb, dim, N):
    """boundaryConditions + riemannSolverLinear on boundary faces
    (ADERDGSolver.cpp:2893-2962): outflow and rigid wall, every face index,
    against the oracle and the reference's kernels compiled from source"""
    rng = np.random.default_rng(31 * dim + N)
    s = eb.Solver(dim, N, eb.PDE_ELASTIC)
    b = N + 1
    F, D2, n = b ** (dim - 1), 2 * dim, 9
    qb = np.stack([random_elastic(rng, 1, D2 * F).reshape(D2, F, 12) for _ in range(n)])
    fb = rng.normal(size=(n, D2, F, 9))
    bc = np.arange(n, dtype=np.int32) % n
    bf = (np.arange(n) % D2).astype(np.int32)
    impls = ["oracle"] + (["ref"] if pyoracle.ref_available(dim) else [])
    for kind in (eb.BC_OUTFLOW, eb.BC_REFLECTIVE):
        fbd = dev(fb)
        s.boundary_conditions(dev(qb), fbd, dev(bc, torch.int32), dev(bf, torch.int32), n, kind)
        got = host(fbd)
        for impl in impls:
            k = pyoracle.Kernels(dim, N, pde=2, impl=impl)
            exp = fb.copy()
            for c, f in zip(bc, bf):
                exp[c, f] = k.lin_boundary_face(fb[c, f], qb[c, f], int(f), 1 if kind == eb.BC_REFLECTIVE else 0).reshape(F, 9)
            assert rel(got, exp) < RTOL, (impl, kind)
        touched = np.zeros((n, D2), bool)
        touched[bc, bf] = True
        assert np.array_equal(got[~touched], fb[~touched])  # other faces untouched
        if kind == eb.BC_OUTFLOW:
            assert np.abs(got[touched]).max() == 0.0  # no jump, no fluctuation
        else:
            assert np.abs(got[touched]).max() > 0.1


BCS = [(2, 4, (12, 12), "outflow", 12), (2, 3, (10, 8), "mixed", 12), (3, 3, (5, 5, 5), "wall", 5),
       (3, 5, (4, 4, 4), "mixed", 3)]


def bc_list(name, dim):
    if name == "outflow":
        return [0] * (2 * dim)
    if name == "wall":
        return [1] * (2 * dim)
    return ([1, 1, 0, 1, -1, -1])[:2 * dim]  # x walls, y outflow / wall, z periodic


@pytest.mark.parametrize("dim,N,cells,bcname,steps", BCS)
def test_elastic_mesh_boundaries_vs_oracle(eb, dim, N, cells, bcname, steps):
    """elastic waves on uniform meshes with outflow and rigid-wall faces,
    against the oracle and the reference's kernels"""
    from exahype_b200 import problems
    bc = bc_list(bcname, dim)
    code = {-1: eb.BC_PERIODIC, 0: eb.BC_OUTFLOW, 1: eb.BC_REFLECTIVE}
    u, _ = problems.elastic_pulse(dim, N, cells, seed=13)
    s = eb.Solver(dim, N, eb.PDE_ELASTIC)
    m = eb.Mesh(s, cells, [0.0] * dim, [1.0] * dim, [code[k] for k in bc])
    m.set_solution(u)
    m.init(0.0)
    m.step(steps)
    a, sa = m.get_solution(), m.state()
    impls = ["oracle"] + (["ref"] if pyoracle.ref_available(dim) else [])
    for impl in impls:
        o = pyoracle.Mesh(dim, N, cells, [1.0] * dim, bc, pde=2, impl=impl, nthreads=8)
        o.set_solution(u)
        o.init(0.0)
        o.step(steps)
        b_, sb = o.get_solution(), o.state()
        assert np.linalg.norm(a - b_) / np.linalg.norm(b_) < RTOL, impl
        assert sa["steps"] == sb["steps"] == steps and sa["dt"] == sb["dt"], impl
    assert np.array_equal(a[..., 9:], u[..., 9:])


def test_refined_elastic_mesh_with_walls_vs_oracle(eb):
    """a refined elastic mesh whose domain faces are rigid walls (x) and
    outflow (y): the boundary faces of the coarse cells"""
    from exahype_b200 import problems
    dim, N, cells, lo, hi, steps = 2, 3, (7, 7), (2, 2), (5, 5), 6
    u = problems.elastic_pulse_refined(dim, N, cells, lo, hi, seed=4)
    s = eb.Solver(dim, N, eb.PDE_ELASTIC)
    m = eb.Mesh.nested(s, cells, [0.0] * dim, [1.0] * dim, [(lo, hi)],
                       bc=[eb.BC_REFLECTIVE, eb.BC_REFLECTIVE, eb.BC_OUTFLOW, eb.BC_OUTFLOW])
    o = pyoracle.RefinedMesh(dim, N, cells, [1.0] * dim, lo, hi, pde=2, bc=[1, 1, 0, 0])
    m.set_solution(u)
    o.set_solution(u)
    m.init(0.0)
    o.init(0.0)
    m.step(steps)
    o.step(steps)
    a, b = m.get_solution(), o.get_solution()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-12
    assert m.state()["steps"] == o.state()["steps"] == steps
