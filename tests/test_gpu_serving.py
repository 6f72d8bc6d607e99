"""Serving with continuous batching (exahype_b200.serving): requests that
arrive while others run are admitted by memory budget, share the batch (or
run on their own limiter stream) and each result equals the request's
standalone run bit for bit."""
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


def small_stream(seed):
    from exahype_b200 import serving
    return serving.request_stream(14, 200.0, seed=seed, sides_2d=(6, 16), sides_3d=(3, 6), orders=(3, 5),
                                  p_limiter=0.3, steps=(3, 12))


def test_served_results_equal_standalone(eb):
    from exahype_b200 import serving
    variants = {(d, o): 0 for d in (2, 3) for o in (3, 5)}
    reqs = small_stream(11)
    kinds = {r.kind for r in reqs}
    assert kinds == {"explosion", "pulse"}
    # a budget of about three requests: later arrivals wait for memory
    budget = 3 * max(serving.Server(1, variants).bytes_for(r) for r in reqs)
    srv = serving.Server(budget, variants)
    done, rejected = srv.run(reqs)
    assert not rejected and all(r.finished is not None for r in done)
    alone = serving.run_one_at_a_time(small_stream(11), variants)
    for a, b in zip(sorted(done, key=lambda r: r.rid), sorted(alone, key=lambda r: r.rid)):
        assert (a.rid, a.kind, a.cells, a.order, a.steps) == (b.rid, b.kind, b.cells, b.order, b.steps)
        assert np.isfinite(b.result).all()
        assert np.array_equal(a.result, b.result), "request %d (%s) differs in the mix" % (a.rid, a.kind)
        assert a.state["steps"] == b.state["steps"] == a.steps
        assert a.state["t"] == b.state["t"]


def test_over_budget_request_is_rejected(eb):
    from exahype_b200 import serving
    reqs = small_stream(3)[:4]
    srv = serving.Server(1, {(d, o): 0 for d in (2, 3) for o in (3, 5)})
    done, rejected = srv.run(reqs)
    assert len(rejected) == 4 and all(r.finished is None for r in done)
