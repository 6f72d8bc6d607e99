"""GPU parity of the point-source path (EXA_PDE_ELASTIC_POINT_SOURCE: the
kernel tests' elastic-wave PDE with a Ricker-wavelet point source) through
the C ABI, against the oracle (1e-12) and against the reference's own
pointSource + spaceTimePredictorLinear<usePointSource = true> compiled from
its sources (oracle/_ref; 5e-11, the precision of the reference's
15-digit basis-function coefficients).

Covered: the predictor kernel with its time averages on cells that hold the
source, cells beside it and a cell whose face carries it; the entry points'
argument checks; uniform meshes (periodic, outflow, rigid walls, a source on
the corner of four cells), fused time stepping, a refined mesh with the
source in the refined box, and the mesh offset."""
import numpy as np
import pytest

import pyoracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

RTOL, REF_TOL = 1e-12, 5e-11
PS = (0.43, 0.57, 0.52, 0.02, 10.0, 1.0)  # x0[3], t0, f0, amplitude


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


def solver(eb, dim, N, ps=PS):
    s = eb.Solver(dim, N, eb.PDE_ELASTIC_POINT_SOURCE)
    s.set_point_source(ps[:dim], *ps[3:])
    return s


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("dim,N", [(2, 3), (2, 5), (3, 3), (3, 5)])
def test_predictor_vs_oracle_and_reference(eb, dim, N, variant):
    rng = np.random.default_rng(dim * 13 + N)
    s = solver(eb, dim, N)
    s.variant = variant
    b = N + 1
    P, F = b ** dim, b ** (dim - 1)
    dx = [0.1, 0.12, 0.09][:dim]
    # cells: the source's, two beside it, one whose right x-face carries it,
    # then cells far away
    centres = [[0.47, 0.52, 0.5], [0.57, 0.52, 0.5], [0.47, 0.64, 0.5], [0.38, 0.55, 0.51]]
    centres += [[0.1 + 0.07 * i, 0.2, 0.3] for i in range(9)]
    centres = np.array(centres)[:, :dim]
    n = len(centres)
    c3 = np.zeros((n, 3))
    c3[:, :dim] = centres
    u = random_elastic(rng, n, P)
    t, dt = 0.012, 3e-3
    qb, fb, du = zeros(n * 2 * dim * F * 12), zeros(n * 2 * dim * F * 9), zeros(n * P * 9)
    qh, fh = zeros(n * P * 12), zeros(n * dim * P * 9)
    s.space_time_predictor_linear_point_source(dev(u), qb, fb, du, dev([t]), dev([dt]), dx, dev(c3), n, lQhi=qh,
                                               lFhi=fh)
    got = dict(lQhbnd=host(qb).reshape(n, -1), lFhbnd=host(fb).reshape(n, -1), lduh=host(du).reshape(n, -1),
               lQhi=host(qh).reshape(n, -1), lFhi=host(fh).reshape(n, -1))
    impls = [("oracle", RTOL)] + ([("ref", REF_TOL)] if pyoracle.ref_available(dim) else [])
    for impl, tol in impls:
        k = pyoracle.Kernels(dim, N, 4, impl=impl, point_source=PS)
        for c in range(n):
            o = k.lin_predictor_at(u[c], dx, dt, centres[c], t)
            for key in got:
                assert rel(got[key][c], o[key]) < tol, (impl, c, key, rel(got[key][c], o[key]))
    # the source changes its cells and only those
    plain = pyoracle.Kernels(dim, N, 2)
    assert rel(got["lduh"][0], plain.lin_predictor(u[0], dx, dt)["lduh"]) > 1e-3
    assert rel(got["lduh"][3], plain.lin_predictor(u[3], dx, dt)["lduh"]) > 1e-3
    assert rel(got["lduh"][5], plain.lin_predictor(u[5], dx, dt)["lduh"]) < RTOL


def test_api_errors(eb):
    s = solver(eb, 2, 3)
    x = zeros(4)
    with pytest.raises(eb.ExaError):
        s.space_time_predictor_linear(x, x, x, x, x, [1, 1], 1)  # the plain entry point rejects it
    with pytest.raises(eb.ExaError):
        s.space_time_predictor_linear_temps(x, x, x, x, x, [1, 1], 1, x, x)
    with pytest.raises(eb.ExaError):  # centres are required
        s.space_time_predictor_linear_point_source(x, x, x, x, x, x, [1, 1], None, 1)
    e = eb.Solver(2, 3, eb.PDE_ELASTIC)
    with pytest.raises(eb.ExaError):
        e.set_point_source([0.5, 0.5])  # no point source in this PDE
    with pytest.raises(eb.ExaError):
        e.space_time_predictor_linear_point_source(x, x, x, x, x, x, [1, 1], x, 1)
    with pytest.raises(eb.ExaError):
        s.set_point_source([0.5, 0.5], t0=float("nan"))


BC_CODE = {-1: -1, 0: 0, 1: 1}
MESHES = [(2, 3, (8, 8), -1, 12, (0.43, 0.57, 0.5)), (2, 5, (6, 6), 0, 6, (0.5, 0.5, 0.5)),
          (2, 3, (10, 8), [1, 1, 0, 0], 10, (0.23, 0.61, 0.5)), (3, 3, (4, 4, 4), 1, 4, (0.43, 0.57, 0.52)),
          (3, 5, (3, 3, 3), -1, 3, (0.43, 0.57, 0.52))]


@pytest.mark.parametrize("dim,N,cells,bc,steps,x0", MESHES)
def test_mesh_vs_oracle_and_reference(eb, dim, N, cells, bc, steps, x0):
    from exahype_b200 import problems
    u, _ = problems.elastic_pulse(dim, N, cells, seed=21)
    u[..., :9] *= 0.1
    ps = tuple(x0) + PS[3:]
    s = solver(eb, dim, N, ps)
    m = eb.Mesh(s, cells, [0.0] * dim, [1.0] * dim, bc)
    m.set_solution(u)
    m.init(0.0)
    m.step(steps)
    a, sa = m.get_solution(), m.state()
    impls = [("oracle", RTOL)] + ([("ref", REF_TOL)] if pyoracle.ref_available(dim) else [])
    for impl, tol in impls:
        o = pyoracle.Mesh(dim, N, cells, [1.0] * dim, bc, pde=4, impl=impl, nthreads=8, point_source=ps)
        o.set_solution(u)
        o.init(0.0)
        o.step(steps)
        b_, sb = o.get_solution(), o.state()
        assert np.linalg.norm(a - b_) / np.linalg.norm(b_) < tol, impl
        assert sa["steps"] == sb["steps"] == steps and sa["dt"] == sb["dt"] and sa["t"] == sb["t"], impl
    assert np.array_equal(a[..., 9:], u[..., 9:])


def test_fused_mesh_vs_oracle(eb):
    """fused time stepping: the predictor after the update starts from the
    predictor time stamp, a rerun from the corrector's"""
    from exahype_b200 import problems
    dim, N, cells, steps = 2, 3, (8, 8), 12
    u, _ = problems.elastic_pulse(dim, N, cells, seed=22)
    u[..., :9] *= 0.1
    s = solver(eb, dim, N)
    m = eb.Mesh(s, cells, [0.0] * dim, [1.0] * dim, eb.BC_PERIODIC)
    m.set_solution(u)
    m.init_fused(0.0, 0.99)
    m.step(steps)
    o = pyoracle.Mesh(dim, N, cells, [1.0] * dim, -1, pde=4, nthreads=8, point_source=PS)
    o.set_solution(u)
    o.init_fused(0.0, 0.99)
    o.step(steps)
    a, b = m.get_solution(), o.get_solution()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < RTOL
    assert m.state()["t"] == o.state()["t"]


def test_refined_mesh_vs_oracle(eb):
    from exahype_b200 import problems
    cells, lo, hi, steps = (7, 7), (2, 2), (5, 5), 5
    u = problems.elastic_pulse_refined(2, 3, cells, lo, hi, seed=4)
    u[..., :9] *= 0.1
    ps = (0.5, 0.45, 0.0) + PS[3:]  # inside the refined box
    s = solver(eb, 2, 3, ps)
    m = eb.Mesh.refined(s, cells, [0.0, 0.0], [1.0, 1.0], lo, hi)
    o = pyoracle.RefinedMesh(2, 3, cells, [1.0, 1.0], lo, hi, pde=4, point_source=ps)
    m.set_solution(u)
    o.set_solution(u)
    m.init(0.0)
    o.init(0.0)
    m.step(steps)
    o.step(steps)
    a, b = m.get_solution(), o.get_solution()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < RTOL
    assert m.state()["steps"] == o.state()["steps"] == steps


def test_mesh_offset(eb):
    """the same problem shifted: a mesh at offset (0.25, -0.5) with the source
    moved by the offset gives the unshifted mesh's solution"""
    from exahype_b200 import problems
    dim, N, cells, steps = 2, 3, (8, 8), 8
    u, _ = problems.elastic_pulse(dim, N, cells, seed=23)
    u[..., :9] *= 0.1
    out = []
    for off in ((0.0, 0.0), (0.25, -0.5)):
        ps = (PS[0] + off[0], PS[1] + off[1], 0.0) + PS[3:]
        m = eb.Mesh(solver(eb, dim, N, ps), cells, list(off), [1.0] * dim, eb.BC_OUTFLOW)
        m.set_solution(u)
        m.init(0.0)
        m.step(steps)
        out.append(m.get_solution())
    assert np.linalg.norm(out[0] - out[1]) / np.linalg.norm(out[0]) < 1e-12
