"""Edge cases of the batched C-ABI kernels on the GPU: empty batches touch
nothing, negative counts are argument errors, ragged and permuted cell lists
give each listed cell exactly its own result (the reference calls the
kernels once per cell, so the order of a batch cannot matter), and the
corrector's min-reduction over a list sees only the listed cells."""
import numpy as np
import pytest

import pyoracle

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eb():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import exahype_b200
    exahype_b200.load()
    return exahype_b200


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def states(rng, n, P):
    u = np.zeros((n, P, 5))
    u[..., 0] = 1.0 + 0.3 * rng.random((n, P))
    u[..., 1:4] = 0.2 * (rng.random((n, P, 3)) - 0.5)
    u[..., 4] = 2.5 + 0.5 * rng.random((n, P))
    return u


def test_empty_batches_touch_nothing(eb):
    s = eb.Solver(3, 3)
    P, F = 64, 16
    u = dev(np.ones((2, P, 5)))
    qb = torch.full((2 * 6 * F * 5,), np.nan, device="cuda", dtype=torch.float64)
    fb = torch.full_like(qb, np.nan)
    du = torch.full((2 * P * 5,), np.nan, device="cuda", dtype=torch.float64)
    dt = dev([1e-3])
    s.space_time_predictor(u, qb, fb, du, dt, [0.1] * 3, 0)
    idx = dev(np.zeros(1), torch.int32)
    s.riemann_solver(qb, fb, idx, idx, idx, 0)
    dmin = dev([1.5])
    s.corrector(u, du, fb, dt, dmin, [0.1] * 3, 0)
    torch.cuda.synchronize()
    assert torch.isnan(qb).all() and torch.isnan(fb).all() and torch.isnan(du).all()
    assert dmin.item() == 1.5


def test_negative_counts_are_errors(eb):
    s = eb.Solver(2, 3)
    buf = dev(np.zeros(4096))
    idx = dev(np.zeros(4), torch.int32)
    with pytest.raises(eb.ExaError):
        s.space_time_predictor(buf, buf, buf, buf, buf, [0.1, 0.1], -1)
    with pytest.raises(eb.ExaError):
        s.riemann_solver(buf, buf, idx, idx, idx, -3)


@pytest.mark.parametrize("variant", [0, 2])
def test_permuted_ragged_cell_list(eb, variant):
    """a list of 37 of 50 cells in scrambled order: every listed cell gets
    its own oracle result, bit for bit the same as in a forward list"""
    rng = np.random.default_rng(11)
    s = eb.Solver(2, 5)
    s.variant = variant
    n, P, F = 50, 36, 6
    u = states(rng, n, P)
    lst = rng.permutation(n)[:37].astype(np.int32)
    outs = []
    for order in (lst, np.sort(lst)):
        qb = torch.full((n * 4 * F * 5,), -7.0, device="cuda", dtype=torch.float64)
        fb = torch.zeros_like(qb)
        du = torch.zeros(n * P * 5, device="cuda", dtype=torch.float64)
        s.space_time_predictor(dev(u), qb, fb, du, dev([2e-3]), [0.04, 0.04], len(order),
                               cell_list=dev(order, torch.int32))
        torch.cuda.synchronize()
        outs.append((qb.cpu().numpy().reshape(n, -1), du.cpu().numpy().reshape(n, -1)))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    k = pyoracle.Kernels(2, 5)
    qb, du = outs[0]
    for c in range(n):
        if c in lst:
            o = k.predictor(u[c], [0.04, 0.04], 2e-3)
            assert np.max(np.abs(qb[c] - o["lQhbnd"])) <= 1e-12 * np.max(np.abs(o["lQhbnd"]))
            assert np.max(np.abs(du[c] - o["lduh"])) <= 1e-12 * np.max(np.abs(o["lduh"]))
        else:
            assert np.all(qb[c] == -7.0)


def test_corrector_min_over_a_list(eb):
    """the admissible step is reduced over the listed cells only; unlisted
    cells keep their solution"""
    rng = np.random.default_rng(5)
    s = eb.Solver(2, 3)
    n, P, F = 40, 16, 4
    u = states(rng, n, P)
    u[7, :, 1] = 3.0  # a fast cell that is not listed
    lst = np.array([0, 3, 9, 10, 22, 39], dtype=np.int32)
    luh = dev(u)
    du = dev(rng.normal(size=(n, P * 5)) * 1e-2)
    fb = dev(rng.normal(size=(n, 4 * F * 5)) * 1e-2)
    dmin = dev([0.0])
    eb.Solver.reset_min(dmin)
    s.corrector(luh, du, fb, dev([1e-4]), dmin, [0.05, 0.05], len(lst), cell_list=dev(lst, torch.int32))
    torch.cuda.synchronize()
    got = luh.cpu().numpy()
    k = pyoracle.Kernels(2, 3)
    dts = []
    for c in range(n):
        if c in lst:
            d = k.surface_integral(du.cpu().numpy()[c], fb.cpu().numpy()[c], [0.05, 0.05])
            ref = k.solution_update(u[c], d, 1e-4).reshape(P, 5)
            assert np.max(np.abs(got[c] - ref)) <= 1e-12 * np.max(np.abs(ref))
            dts.append(k.stable_dt(got[c], [0.05, 0.05]))  # bit-identical from the same solution
        else:
            assert np.array_equal(got[c], u[c])
    assert dmin.item() == min(dts)


def test_nan_in_the_input_is_a_status(eb):
    """a non-finite value planted in the host-prepared input is reported by
    exa_mesh_validate, stepping goes on without a trap (the step-size
    minimum skips NaN, as std::min in the reference does) and the NaN
    spreads to the neighbours; a clean mesh reports 0"""
    from exahype_b200 import problems
    u, _ = problems.gaussian_pulse_2d(3, (8, 8), seed=0)
    s = eb.Solver(2, 3)
    m = eb.Mesh(s, (8, 8), [0.0, 0.0], [1.0, 1.0], eb.BC_PERIODIC)
    m.set_solution(u)
    m.init(0.0)
    m.step(2)
    assert m.validate() == 0
    bad = u.copy()
    bad[13, 5, 4] = np.nan
    m.set_solution(bad)
    m.init(0.0)
    n0 = m.validate()
    assert n0 >= 1
    assert np.isfinite(m.state()["dt"]) and m.state()["dt"] > 0
    assert m.run_until(1.0, max_steps=3) == 3
    assert m.validate() > n0


def test_step_size_skips_non_finite_nodes_in_every_block(eb):
    """stableTimeStepSize keeps dt = std::min(dt, CFL PNPM / den) from
    DBL_MAX: a node whose denominator is NaN (negative pressure, a NaN
    value) never replaces the minimum. With such a node in every block of
    the launch, the mesh step size is still the minimum over all finite
    nodes, equal to the oracle's"""
    from exahype_b200 import problems
    u, _ = problems.gaussian_pulse_2d(3, (8, 8), seed=1)
    bad = u.copy()
    for c in range(0, 64, 5):  # every 16-cell block gets several
        bad[c, (3 * c) % 16, 4] = -1.0  # negative energy: negative pressure, NaN sound speed
    s = eb.Solver(2, 3)
    m = eb.Mesh(s, (8, 8), [0.0, 0.0], [1.0, 1.0], eb.BC_PERIODIC)
    m.set_solution(bad)
    m.init(0.0)
    k = pyoracle.Kernels(2, 3, pde=0)
    exp = min(k.stable_dt(bad[c], [0.125, 0.125]) for c in range(64))
    assert np.isfinite(exp) and m.state()["dt"] == exp
