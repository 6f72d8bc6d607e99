"""GPU parity of the source and non-conservative-product paths (useSource =
useNCP = true; EXA_PDE_EULER_SOURCE_NCP: the kernel tests' Euler mock with
an algebraic source and the tests' non-zero product mock) against the oracle
and against the reference's own templates compiled from its sources with
the same flags (oracle/_ref), through the C ABI.

Covered: the predictor's source branch with the gradients of the iterate
(3d/spaceTimePredictorNonlinear.cpph:238-276, 2d :180-211) and its
temporaries (the source block of lFi and lFhi), the volume integral's
time-averaged source, the Riemann solver's fluctuations on interior faces
and on boundary faces (3d/riemannSolverNonlinear.cpph:92-110), and
uniform-mesh runs. Bar: 1e-12 relative, equal Picard sweep counts.
"""
import numpy as np
import pytest

import pyoracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

RTOL = 1e-12


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


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def states(rng, shape):
    u = np.zeros(shape + (6,))
    u[..., 0] = 1.0 + 0.2 * rng.random(shape)
    u[..., 1:4] = 0.2 * (rng.random(shape + (3,)) - 0.5)
    u[..., 4] = 2.5 + 0.3 * rng.random(shape)
    u[..., 5] = rng.random(shape)
    return u


@pytest.mark.parametrize("dim,order", [(2, 3), (2, 5), (3, 3), (3, 5)])
def test_predictor_temporaries_vs_oracle_and_reference(eb, dim, order):
    rng = np.random.default_rng(dim * 10 + order)
    s = eb.Solver(dim, order, eb.PDE_EULER_SOURCE_NCP)
    b = order + 1
    P, F, nV, nD = b ** dim, b ** (dim - 1), 5, 6
    luh = states(rng, (P,))
    dx = [0.05, 0.04, 0.045][:dim]
    dt = 1e-3
    z = lambda n: torch.zeros(n, device="cuda", dtype=torch.float64)
    qb, fb, du = z(2 * dim * F * nD), z(2 * dim * F * nV), z(P * nV)
    lQi, lFi, lQhi, lFhi = z(P * b * nD), z(P * b * (dim + 1) * nV), z(P * nD), z(P * (dim + 1) * nV)
    it = torch.zeros(1, device="cuda", dtype=torch.int32)
    s.space_time_predictor_temps(dev(luh), qb, fb, du, dev([dt]), dx, 1, it, lQi, lFi, lQhi, lFhi)
    got = dict(lQi=host(lQi), lFi=host(lFi), lQhi=host(lQhi), lFhi=host(lFhi), lQhbnd=host(qb), lFhbnd=host(fb),
               lduh=host(du))
    for impl in ("oracle", "ref"):
        o = pyoracle.Kernels(dim, order, pde=3, impl=impl).predictor(luh, dx, dt, temps=True)
        assert host(it)[0] == o["iterations"], impl
        for key, val in got.items():
            assert rel(val, o[key]) < RTOL, (impl, key, rel(val, o[key]))
    # the source block is live: lFhi's last block and lduh differ from the plain mock's
    assert np.abs(got["lFhi"].reshape(dim + 1, P, nV)[dim]).max() > 0.1


@pytest.mark.parametrize("variant", [0, 3])
@pytest.mark.parametrize("dim,order", [(2, 5), (3, 3)])
def test_predictor_batch_vs_oracle(eb, dim, order, variant):
    rng = np.random.default_rng(3 + dim + order)
    s = eb.Solver(dim, order, eb.PDE_EULER_SOURCE_NCP)
    s.variant = variant
    b = order + 1
    P, F, nV, nD = b ** dim, b ** (dim - 1), 5, 6
    n = 29
    u = states(rng, (n, P))
    dx = [0.05, 0.04, 0.045][:dim]
    dt = 5e-4
    qb = torch.zeros(n * 2 * dim * F * nD, device="cuda", dtype=torch.float64)
    fb = torch.zeros(n * 2 * dim * F * nV, device="cuda", dtype=torch.float64)
    du = torch.zeros(n * P * nV, device="cuda", dtype=torch.float64)
    it = torch.zeros(n, device="cuda", dtype=torch.int32)
    s.space_time_predictor(dev(u), qb, fb, du, dev([dt]), dx, n, iterations=it)
    qb, fb, du, it = host(qb).reshape(n, -1), host(fb).reshape(n, -1), host(du).reshape(n, -1), host(it)
    k = pyoracle.Kernels(dim, order, pde=3)
    for c in range(0, n, 4):
        o = k.predictor(u[c], dx, dt)
        assert it[c] == o["iterations"]
        assert rel(qb[c], o["lQhbnd"]) < RTOL
        assert rel(fb[c], o["lFhbnd"]) < RTOL
        assert rel(du[c], o["lduh"]) < RTOL


@pytest.mark.parametrize("dim,order", [(2, 3), (3, 5)])
def test_riemann_and_boundary_fluctuations(eb, dim, order):
    rng = np.random.default_rng(dim * 7 + order)
    s = eb.Solver(dim, order, eb.PDE_EULER_SOURCE_NCP)
    b = order + 1
    F, nV, nD, D2 = b ** (dim - 1), 5, 6, 2 * dim
    n = 11
    qb = states(rng, (n, D2, F))
    fb = rng.standard_normal((n, D2, F, nV))
    fl = np.array([0, 1, 2, 5, 9], dtype=np.int32)
    fr = np.array([1, 2, 3, 6, 0], dtype=np.int32)
    fd = np.array([0, 1, dim - 1, 0, 1], dtype=np.int32)
    fbd = dev(fb)
    s.riemann_solver(dev(qb), fbd, dev(fl, torch.int32), dev(fr, torch.int32), dev(fd, torch.int32), len(fl))
    bc = np.array([4, 7, 8, 10], dtype=np.int32)
    bf = np.array([0, 2 * dim - 1, 3, 2], dtype=np.int32)
    s.boundary_conditions(dev(qb), fbd, dev(bc, torch.int32), dev(bf, torch.int32), len(bc), eb.BC_OUTFLOW)
    got = host(fbd).reshape(n, D2, F, nV)
    for impl in ("oracle", "ref"):
        k = pyoracle.Kernels(dim, order, pde=3, impl=impl)
        exp = fb.copy()
        for l, r, d in zip(fl, fr, fd):
            FL, FR = k.riemann(exp[l, 2 * d + 1], exp[r, 2 * d], qb[l, 2 * d + 1], qb[r, 2 * d], int(d))
            exp[l, 2 * d + 1] = FL.reshape(F, nV)
            exp[r, 2 * d] = FR.reshape(F, nV)
        for c, f in zip(bc, bf):
            exp[c, f] = k.boundary_face(exp[c, f], qb[c, f], int(f)).reshape(F, nV)
        assert rel(got, exp) < RTOL, impl
    # the fluctuations differ between the two sides of a face
    assert np.abs(got[0, 1] - got[1, 0]).max() > 0.1


@pytest.mark.parametrize("dim,order,cells,bc,steps", [(2, 3, (8, 8), -1, 5), (2, 5, (6, 6), 0, 3),
                                                      (3, 3, (4, 4, 4), -1, 3)])
def test_mesh_vs_oracle_and_reference(eb, dim, order, cells, bc, steps):
    from exahype_b200 import problems
    if dim == 2:
        u, _ = problems.gaussian_pulse_2d(order, cells, seed=11)
    else:
        u, _ = problems.gaussian_pulses_3d(order, cells, seed=11)
    u6 = np.concatenate([u, np.zeros(u.shape[:-1] + (1,))], axis=-1)
    s = eb.Solver(dim, order, eb.PDE_EULER_SOURCE_NCP)
    m = eb.Mesh(s, cells, [0.0] * dim, [1.0] * dim, bc)
    m.set_solution(u6)
    m.init(0.0)
    m.step(steps)
    a, sa = m.get_solution(), m.state()
    for impl in ("oracle", "ref"):
        o = pyoracle.Mesh(dim, order, cells, [1.0] * dim, bc, pde=3, impl=impl, nthreads=8)
        o.set_solution(u6)
        o.init(0.0)
        o.step(steps)
        b_, sb = o.get_solution(), o.state()
        assert np.linalg.norm(a - b_) / np.linalg.norm(b_) < RTOL, impl
        assert sa["steps"] == sb["steps"] == steps and sa["picard_sweeps"] == sb["picard_sweeps"], (impl, sa, sb)
        assert abs(sa["t"] - sb["t"]) <= 1e-13 * sb["t"]
