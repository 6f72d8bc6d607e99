"""The oracle's point-source path (pde 4: the kernel tests' elastic-wave PDE
with a Ricker-wavelet point source) against the reference's own templates
compiled from its sources (oracle/_ref): pointSource
(c/{2d,3d}/pointSource.cpph), spaceTimePredictorLinear<usePointSource =
true> and uniform / refined mesh runs. CPU only.

Bar: 5e-11 relative against the reference. The reference's basis functions
(kernels/DGBasisFunctions.cpp) are products of linear factors written with 15
significant digits, the oracle's the exact Lagrange products of the
Gauss-Legendre nodes; near a factor's root the truncation shows at 1e-12 in
the projected source and up to 1e-11 in the predictor's outputs (3D, N = 5)."""
import numpy as np
import pytest

import pyoracle
from exahype_b200 import problems

pytestmark = pytest.mark.skipif(not (pyoracle.ref_available(2) and pyoracle.ref_available(3)),
                                reason="oracle/_ref not built")

TOL = 5e-11
PS = (0.43, 0.57, 0.52, 0.02, 10.0, 1.0)  # x0[3], t0, f0, amplitude


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def random_elastic(rng, n):
    return np.concatenate([rng.normal(size=(n, 9)), rng.uniform(1, 3, size=(n, 1)), rng.uniform(0.5, 1.5, size=(n, 1)),
                           rng.uniform(1, 2, size=(n, 1))], axis=1)


@pytest.mark.parametrize("dim,N", [(2, 3), (2, 5), (3, 3), (3, 5)])
def test_point_source_kernel(dim, N):
    o = pyoracle.Kernels(dim, N, 4, point_source=PS)
    r = pyoracle.Kernels(dim, N, 4, impl="ref", point_source=PS)
    dx = [0.1, 0.12, 0.09][:dim]
    t, dt = 0.015, 0.004
    # a cell holding the source, one beside it, one whose face carries it
    inside = [0.47, 0.52, 0.5][:dim]
    outside = [0.2, 0.3, 0.4][:dim]
    on_face = [0.43 - 0.05, 0.55, 0.51][:dim]  # x0[0] on the cell's right face
    a, b = o.point_source(t, dt, inside, dx), r.point_source(t, dt, inside, dx)
    assert a.shape == (N + 2, (N + 1) ** dim, 9)
    assert rel(a, b) < TOL
    assert np.abs(a[:, :, :3]).max() > 1.0 and np.abs(a[:, :, 3:]).max() == 0.0  # normal stresses only
    assert np.abs(o.point_source(t, dt, outside, dx)).max() == 0.0
    assert np.abs(r.point_source(t, dt, outside, dx)).max() == 0.0
    a, b = o.point_source(t, dt, on_face, dx), r.point_source(t, dt, on_face, dx)
    assert rel(a, b) < TOL and np.abs(a).max() > 0.0  # the closed box: a source on the face counts


@pytest.mark.parametrize("dim,N", [(2, 3), (2, 5), (3, 3), (3, 5)])
def test_predictor_with_point_source(dim, N):
    rng = np.random.default_rng(dim * 17 + N)
    o = pyoracle.Kernels(dim, N, 4, point_source=PS)
    r = pyoracle.Kernels(dim, N, 4, impl="ref", point_source=PS)
    u = random_elastic(rng, (N + 1) ** dim)
    dx = [0.1, 0.12, 0.09][:dim]
    centre = [0.47, 0.52, 0.5][:dim]
    a = o.lin_predictor_at(u, dx, 3e-3, centre, 0.01)
    b = r.lin_predictor_at(u, dx, 3e-3, centre, 0.01)
    for key in a:
        assert rel(a[key], b[key]) < TOL, key
    plain = o.lin_predictor(u, dx, 3e-3)
    assert rel(a["lduh"], plain["lduh"]) > 1e-3  # the source is live
    far = o.lin_predictor_at(u, dx, 3e-3, [0.1, 0.1, 0.1][:dim], 0.01)
    for key in far:
        assert np.array_equal(far[key], plain[key]), key  # and absent outside its cell


@pytest.mark.parametrize("dim,N,cells,bc,steps,x0", [(2, 3, (8, 8), -1, 10, (0.43, 0.57, 0.5)),
                                                     (2, 5, (6, 6), 0, 6, (0.5, 0.5, 0.5)),
                                                     (3, 3, (4, 4, 4), 1, 4, (0.43, 0.57, 0.52))])
def test_mesh_runs(dim, N, cells, bc, steps, x0):
    """uniform meshes; (0.5, 0.5) sits on the corner of four cells of the 6 x 6
    grid, each of which takes the whole source as the reference's does"""
    u, _ = problems.elastic_pulse(dim, N, cells, seed=9)
    u[..., :9] *= 0.1
    ps = tuple(x0) + PS[3:]
    res = []
    for impl in ("oracle", "ref"):
        m = pyoracle.Mesh(dim, N, cells, [1.0] * dim, bc, pde=4, impl=impl, nthreads=4, point_source=ps)
        m.set_solution(u)
        m.init(0.0)
        m.step(steps)
        res.append((m.get_solution(), m.state()))
    (a, sa), (b, sb) = res
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < TOL
    assert sa["dt"] == sb["dt"] and sa["steps"] == sb["steps"] == steps
    m = pyoracle.Mesh(dim, N, cells, [1.0] * dim, bc, pde=2, nthreads=4)
    m.set_solution(u)
    m.init(0.0)
    m.step(steps)
    assert np.linalg.norm(m.get_solution() - a) / np.linalg.norm(a) > 1e-3


def test_mesh_linearity_and_locality():
    """a linear PDE from rest: the solution scales with the amplitude, and
    after one step only the source's cell and its face neighbours moved"""
    dim, N, cells = 2, 3, (8, 8)
    u, _ = problems.elastic_pulse(dim, N, cells, seed=9)
    u[..., :9] = 0.0
    out = []
    for amp in (1.0, 2.0):
        m = pyoracle.Mesh(dim, N, cells, [1.0] * dim, -1, pde=4, point_source=PS[:5] + (amp,))
        m.set_solution(u)
        m.init(0.0)
        m.step(1)
        out.append(m.get_solution()[..., :9])
    assert np.linalg.norm(out[1] - 2 * out[0]) <= 1e-13 * np.linalg.norm(out[1])
    moved = np.abs(out[0]).reshape(cells[1], cells[0], -1).max(axis=2) > 0
    src = (int(PS[1] * 8), int(PS[0] * 8))  # (y, x) of the source's cell
    for y in range(8):
        for x in range(8):
            near = abs(y - src[0]) + abs(x - src[1]) <= 1
            assert moved[y, x] == near, (y, x)


def test_refined_mesh_vs_reference():
    cells, lo, hi = (7, 7), (2, 2), (5, 5)
    u = problems.elastic_pulse_refined(2, 3, cells, lo, hi, seed=4)
    u[..., :9] *= 0.1
    ps = (0.5, 0.45, 0.0) + PS[3:]  # inside the refined box
    res = []
    for impl in ("oracle", "ref"):
        m = pyoracle.RefinedMesh(2, 3, cells, [1.0, 1.0], lo, hi, pde=4, impl=impl, point_source=ps)
        m.set_solution(u)
        m.init(0.0)
        m.step(4)
        res.append(m.get_solution())
    assert np.linalg.norm(res[0] - res[1]) / np.linalg.norm(res[1]) < TOL
