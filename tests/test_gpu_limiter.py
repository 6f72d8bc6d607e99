"""GPU parity of the a-posteriori subcell limiter against the oracle's limiting
harness, through the C ABI (exa_lmesh_*).

Bar: the limiter status of every cell (the troubled-cell mask and its helper
layers) is identical to the oracle's after every step, and so are the step
count, the number of irregular steps (local recomputations) and the number of
Picard sweeps; time and step size agree to 1e-12 relative; the DG solution to
1e-11 relative L2 and the interior FV subcells of every allocated patch to
1e-11 relative max-norm. (The FV update and the projections are summed in a
different order than the oracle's loops, so the fields differ at round-off
level, never in the discrete decisions.)
"""
import numpy as np
import pytest

import pyoracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-11


@pytest.fixture(scope="module")
def eb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import exahype_b200
    exahype_b200.load()
    return exahype_b200


def rel_l2(a, b):
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


def interior(lim, dim, order):
    """interior subcells of FV patches (n, E^d, 5) -> (n, B^d, 5)"""
    B = 2 * order + 1
    E = B + 4
    n = lim.shape[0]
    if dim == 2:
        return lim.reshape(n, E, E, 5)[:, 2:2 + B, 2:2 + B].reshape(n, -1, 5)
    return lim.reshape(n, E, E, E, 5)[:, 2:2 + B, 2:2 + B, 2:2 + B].reshape(n, -1, 5)


def make_pair(eb, dim, order, cells, bc, helper, cure, seed, fv_ic=True, problem="explosion", radius=0.2,
              variant=None):
    from exahype_b200 import problems
    if problem == "explosion":
        luh, fv, _ = problems.explosion(dim, order, cells, seed=seed, radius=radius)
    else:
        luh, _ = problems.gaussian_pulse_2d(order, cells, seed=seed)
        fv = None
    size = [1.0] * dim
    s = eb.Solver(dim, order)
    if variant is not None:
        s.variant = variant
    g = eb.LimitingMesh(s, cells, [0.0] * dim, size, bc, helper_layers=helper, cure_steps=cure)
    o = pyoracle.LimitingMesh(dim, order, cells, size, bc, helper_layers=helper, cure_steps=cure, nthreads=8)
    for m in (g, o):
        m.set_solution(luh)
        if fv_ic and fv is not None:
            m.set_fv_initial(fv)
        m.init(0.0)
    return s, g, o


def compare(g, o, dim, order, where, check_lim=True):
    sg, so = g.status(), o.status()
    diff = np.nonzero(sg != so)[0]
    assert diff.size == 0, "%s: status differs in %d cells, first %s: gpu %s oracle %s" % (
        where, diff.size, diff[:8].tolist(), sg[diff[:8]].tolist(), so[diff[:8]].tolist())
    a, b = g.state(), o.state()
    assert a["steps"] == b["steps"], where
    assert a["irregular_steps"] == b["irregular_steps"], (where, a, b)
    assert a["picard_sweeps"] == b["picard_sweeps"], (where, a, b)
    assert abs(a["t"] - b["t"]) <= 1e-12 * max(abs(b["t"]), 1e-300), (where, a, b)
    assert abs(a["dt"] - b["dt"]) <= 1e-12 * abs(b["dt"]), (where, a, b)
    e = rel_l2(g.get_solution(), o.get_solution())
    assert e < FIELD_TOL, "%s: DG solution rel L2 %.3e" % (where, e)
    if check_lim:
        lg, ag = g.limiter()
        lo, ao = o.limiter()
        sel = so > 0
        assert np.array_equal(ag[sel] != 0, ao[sel] != 0), where
        if sel.any():
            ig, io = interior(lg[sel], dim, order), interior(lo[sel], dim, order)
            el = np.max(np.abs(ig - io)) / np.max(np.abs(io))
            assert el < FIELD_TOL, "%s: FV subcells rel max %.3e" % (where, el)
    return sg


@pytest.mark.parametrize("dim,order,cells,steps,helper,cure", [
    (2, 3, (20, 20), 40, 1, 0),
    (2, 5, (16, 16), 40, 1, 0),
    (2, 5, (16, 16), 40, 2, 10),
    (2, 4, (14, 14), 30, 1, 2),
    (2, 7, (10, 10), 25, 1, 0),
])
def test_limiting_mesh_2d_outflow(eb, dim, order, cells, steps, helper, cure):
    _, g, o = make_pair(eb, dim, order, cells, 0, helper, cure, seed=3)
    s0 = compare(g, o, dim, order, "init")
    assert (s0 == 2 * helper + 1).any(), "the explosion must start with troubled cells"
    seen_irregular = False
    for k in range(steps):
        g.step(1)
        o.step(1)
        compare(g, o, dim, order, "step %d" % (k + 1), check_lim=(k % 5 == 4))
        seen_irregular |= o.state()["irregular_steps"] > 0
    if helper == 1:  # with one helper layer the shock soon leaves the FV region
        assert seen_irregular


@pytest.mark.parametrize("dim,order,cells,steps,helper,cure", [
    (2, 3, (20, 20), 40, 1, 0),
    (2, 5, (16, 16), 40, 1, 0),
    (2, 4, (14, 14), 30, 1, 2),
])
def test_limiting_mesh_2d_tensor_memory_predictor(eb, dim, order, cells, steps, helper, cure):
    """the same comparison with the line-form predictor that keeps the Picard
    iterate in tensor memory (variant 8), run on the limiting mesh's
    device-compacted cell lists with several cells per block"""
    _, g, o = make_pair(eb, dim, order, cells, 0, helper, cure, seed=3, variant=8)
    compare(g, o, dim, order, "init")
    for k in range(steps):
        g.step(1)
        o.step(1)
        compare(g, o, dim, order, "step %d" % (k + 1), check_lim=(k % 5 == 4))


@pytest.mark.parametrize("order,cells,steps,variant", [(3, (6, 6, 6), 10, None), (5, (5, 5, 5), 6, None),
                                                     (3, (6, 6, 6), 10, 8), (5, (5, 5, 5), 6, 8)])
def test_limiting_mesh_3d_outflow(eb, order, cells, steps, variant):
    """variant 8: the tensor-memory predictor on the limiting mesh's cell lists
    (3D N=5: one cell per block; N=3: four)"""
    _, g, o = make_pair(eb, 3, order, cells, 0, 1, 0, seed=1, variant=variant)
    compare(g, o, 3, order, "init")
    for k in range(steps):
        g.step(1)
        o.step(1)
        compare(g, o, 3, order, "step %d" % (k + 1), check_lim=(k % 3 == 2))


@pytest.mark.parametrize("dim,order,cells,bc,steps,helper,cure", [
    (2, 5, (16, 16), 1, 40, 2, 10),  # the demonstrator's walls, helper layers and cure steps
    (2, 3, (14, 10), [1, 1, 0, 0], 30, 1, 0),
    (3, 3, (5, 5, 5), 1, 8, 1, 0),
    (3, 3, (5, 5, 5), 0, 8, 1, 0),  # outflow: the 3D y-/z-left ghost layers of the reference
])
def test_limiting_mesh_walls_and_boundary_patches(eb, dim, order, cells, bc, steps, helper, cure):
    """a wide explosion whose front reaches every domain face: FV patches on
    boundary cells with reflective walls (the demonstrator's DG and FV
    boundaryValues: normal momentum negated) or outflow"""
    _, g, o = make_pair(eb, dim, order, cells, bc, helper, cure, seed=2, radius=0.45)
    compare(g, o, dim, order, "init")
    fv_on_edge = False
    A = helper + 1
    for k in range(steps):
        g.step(1)
        o.step(1)
        st = compare(g, o, dim, order, "step %d" % (k + 1), check_lim=(k % 3 == 2))
        grid = st.reshape(tuple(reversed(cells)))
        for ax in range(dim):
            for end in (0, -1):
                idx = [slice(None)] * dim
                idx[ax] = end
                fv_on_edge |= bool((grid[tuple(idx)] >= A).any())
    assert fv_on_edge


def test_limiting_mesh_periodic_and_projection_seed(eb):
    """periodic faces (FV halo across the wrap) and patches seeded by projecting
    the DG initial data (no FV initial condition given)"""
    _, g, o = make_pair(eb, 2, 3, (16, 16), -1, 1, 0, seed=5, fv_ic=False)
    compare(g, o, 2, 3, "init")
    for k in range(30):
        g.step(1)
        o.step(1)
        compare(g, o, 2, 3, "step %d" % (k + 1), check_lim=(k % 5 == 4))


def test_limiting_mesh_transient_troubled_pulse(eb):
    """an under-resolved pulse (12x12 cells, N=3) starts admissible everywhere,
    trips the DMP in a few cells on a few steps (irregular changes) and is
    cured again: same statuses and recomputations as the oracle"""
    _, g, o = make_pair(eb, 2, 3, (12, 12), -1, 1, 0, seed=0, problem="pulse")
    assert not g.status().any()
    for k in range(10):
        g.step(1)
        o.step(1)
        compare(g, o, 2, 3, "step %d" % (k + 1))
    assert o.state()["irregular_steps"] > 0


def test_limiting_mesh_run_until(eb):
    """run_until stops on the same step as the oracle (same step count and
    time), with the reference's extra clock advance on irregular steps"""
    _, g, o = make_pair(eb, 2, 5, (12, 12), 0, 1, 0, seed=7)
    n_g = g.run_until(0.02)
    n_o = o.run_until(0.02)
    assert n_g == n_o
    compare(g, o, 2, 5, "t=0.02")


def test_limiting_explosion_81x81_first_steps(eb):
    """2D N=5 explosion on 81x81 outflow cells, DMP delta0 1e-4, eps 1e-3:
    troubled-cell mask identical to the oracle at each of the first 12 steps"""
    _, g, o = make_pair(eb, 2, 5, (81, 81), 0, 1, 0, seed=0)
    compare(g, o, 2, 5, "init", check_lim=False)
    for k in range(12):
        g.step(1)
        o.step(1)
        compare(g, o, 2, 5, "step %d" % (k + 1), check_lim=(k == 11))


def test_limiting_explosion_81x81_to_t02(eb):
    """the full 2D N=5 81x81 explosion to t = 0.2 on the GPU: positivity of
    density and pressure on every node, statuses in range, finite fields"""
    from exahype_b200 import problems
    luh, fv, _ = problems.explosion(2, 5, (81, 81), seed=0)
    s = eb.Solver(2, 5)
    g = eb.LimitingMesh(s, (81, 81), [0.0, 0.0], [1.0, 1.0], 0, helper_layers=1, cure_steps=0)
    g.set_solution(luh)
    g.set_fv_initial(fv)
    g.init(0.0)
    n = g.run_until(0.2)
    st = g.state()
    assert st["t"] >= 0.2 and st["steps"] == n > 100
    u = g.get_solution()
    assert np.isfinite(u).all()
    stat = g.status()
    assert stat.min() >= 0 and stat.max() <= 3 and (stat == 3).any()
    dg = u[stat == 0]  # unlimited cells passed the DMP and admissibility on this step
    rho = dg[..., 0]
    p = 0.4 * (dg[..., 4] - 0.5 * np.sum(dg[..., 1:4] ** 2, axis=-1) / rho)
    assert rho.min() > 0 and p.min() > 0


@pytest.mark.parametrize("dim,order,cells", [(2, 5, (24, 24)), (3, 3, (8, 8, 8))])
def test_run_until_graph_matches_eager_steps(eb, dim, order, cells):
    """run_until replays a captured, device-gated step in chunks; it takes
    exactly the steps an eager loop with a host check of t and dt takes, with
    bit-identical solution, statuses and FV patches, also when max_steps ends
    a chunk early and when the predictor variant changes between calls"""
    from exahype_b200 import problems
    luh, fv, _ = problems.explosion(dim, order, cells, seed=3)
    s = eb.Solver(dim, order)
    meshes = []
    for _ in range(2):
        m = eb.LimitingMesh(s, cells, [0.0] * dim, [1.0] * dim, 0, helper_layers=1, cure_steps=0)
        m.set_solution(luh)
        m.set_fv_initial(fv)
        m.init(0.0)
        meshes.append(m)
    graph, eager = meshes

    def eager_until(t_end, max_steps=10 ** 9):
        n = 0
        while n < max_steps:
            st = eager.state()
            if not (st["t"] < t_end and st["dt"] > 0):
                break
            eager.step(1)
            n += 1
        return n

    assert graph.run_until(0.05, max_steps=5) == eager_until(0.05, max_steps=5) == 5
    s.variant = 1 if s.variant != 1 else 0
    t_end = 0.03 if dim == 2 else 0.06
    n_g, n_e = graph.run_until(t_end), eager_until(t_end)
    assert n_g == n_e > 5
    assert graph.run_until(t_end) == 0  # already there: no replay changes anything
    a, b = graph.state(), eager.state()
    assert a == b and a["irregular_steps"] > 0
    assert np.array_equal(graph.get_solution(), eager.get_solution())
    assert np.array_equal(graph.status(), eager.status())
    la, ma = graph.limiter()
    lb, mb = eager.limiter()
    assert np.array_equal(ma, mb) and np.array_equal(la[ma != 0], lb[mb != 0])
