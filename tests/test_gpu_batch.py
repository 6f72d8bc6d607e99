"""The batched ragged ensemble (exa_batch_*): every instance must compute
exactly what a single Mesh of the same problem computes -- bit for bit, same
step sizes and times -- whatever else is in the batch, with and without the
CUDA graph, and across membership changes between steps."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import exahype_b200
    exahype_b200.load()
    return exahype_b200


def problems_mix():
    from exahype_b200 import problems
    out = []
    for order, cells, bc, seed, amp in [(3, (9, 9), -1, 1, 0.3), (5, (12, 12), -1, 2, 0.5), (7, (9, 9), -1, 3, 0.2),
                                        (3, (14, 10), 0, 4, 0.4), (5, (9, 9), 1, 6, 0.1), (3, (11, 11), -1, 7, 0.45)]:
        luh, _ = problems.gaussian_pulse_2d(order, cells, seed=seed, amplitude=amp)
        if bc == 1:  # reflective walls: a pulse at rest (p = 1), which spreads and reflects
            luh[..., 1:4] = 0.0
            luh[..., 4] = 2.5
        out.append(dict(dim=2, order=order, cells=cells, bc=bc, luh=luh))
    luh, _ = problems.gaussian_pulses_3d(3, (5, 5, 5), seed=5)
    out.append(dict(dim=3, order=3, cells=(5, 5, 5), bc=-1, luh=luh))
    return out


def single(eb, p, steps, variant):
    s = eb.Solver(p["dim"], p["order"])
    s.variant = variant
    m = eb.Mesh(s, p["cells"], [0.0] * p["dim"], [1.0] * p["dim"], p["bc"])
    m.set_solution(p["luh"])
    m.init(0.0)
    m.step(steps)
    return m.get_solution(), m.state()


def check_same(eb, bt, iid, p, steps):
    v = bt.variant(p["dim"], p["order"])
    u, st = single(eb, p, steps, v)
    got = bt.get_solution(iid)
    assert np.isfinite(u).all()
    bs = bt.state(iid)
    assert bs["steps"] == st["steps"] == steps
    assert bs["t"] == st["t"] and bs["dt"] == st["dt"], (bs, st)
    assert np.array_equal(got, u), "instance %d differs from its single-mesh run" % iid


@pytest.mark.parametrize("graph", [True, False])
def test_batch_matches_single_meshes(eb, graph):
    probs = problems_mix()
    bt = eb.Batch()
    bt.set_graph(graph)
    ids = [bt.add(p["dim"], p["order"], p["cells"], [1.0] * p["dim"], p["bc"], p["luh"]) for p in probs]
    bt.step(8)
    for iid, p in zip(ids, probs):
        check_same(eb, bt, iid, p, 8)


def test_batch_tensor_memory_predictor(eb):
    """every order forced to variant 8 (the tensor-memory predictor where the
    shape allows it): each instance still equals its single-mesh run"""
    probs = problems_mix()
    bt = eb.Batch()
    for p in probs:  # before the first instance of each order: its first predictor runs variant 8 too
        bt.set_variant(p["dim"], p["order"], 8)
    ids = [bt.add(p["dim"], p["order"], p["cells"], [1.0] * p["dim"], p["bc"], p["luh"]) for p in probs]
    bt.step(6)
    for iid, p in zip(ids, probs):
        assert bt.variant(p["dim"], p["order"]) == 8
        check_same(eb, bt, iid, p, 6)


def test_batch_membership_changes(eb):
    probs = problems_mix()
    bt = eb.Batch()
    a = bt.add(2, 3, probs[0]["cells"], [1.0, 1.0], -1, probs[0]["luh"])
    b = bt.add(2, 5, probs[1]["cells"], [1.0, 1.0], -1, probs[1]["luh"])
    bt.step(3)
    c = bt.add(2, 3, probs[5]["cells"], [1.0, 1.0], -1, probs[5]["luh"])
    d = bt.add(2, 7, probs[2]["cells"], [1.0, 1.0], -1, probs[2]["luh"])
    bt.step(2)
    bt.remove(a)
    bt.step(3)
    check_same(eb, bt, b, probs[1], 8)
    check_same(eb, bt, c, probs[5], 5)
    check_same(eb, bt, d, probs[2], 5)
    with pytest.raises(eb.ExaError):
        bt.get_solution(a)
    assert bt.device_bytes() > 0
