"""GPU parity of the kernel-level limiter entry points (projections and the
MUSCL-Hancock FV update) against the oracle's per-cell restatement, through
the C ABI. Tolerance 1e-12 relative max-norm (the GPU sums the separable
projections and may contract to FMA; the oracle does neither)."""
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
    q = np.zeros(shape + (5,))
    q[..., 0] = 1.0 + 0.3 * rng.random(shape)
    q[..., 1:4] = 0.2 * (rng.random(shape + (3,)) - 0.5)
    q[..., 4] = 2.5 + 0.5 * rng.random(shape)
    return q


@pytest.mark.parametrize("dim,order", [(2, 3), (2, 5), (2, 7), (3, 3), (3, 5)])
def test_projections_vs_oracle(eb, dim, order):
    rng = np.random.default_rng(10 * dim + order)
    k = pyoracle.Kernels(dim, order)
    n = 37
    E = 2 * order + 5
    luh = states(rng, (n, (order + 1) ** dim))
    sentinel = -7.0
    lim0 = np.full((n, E ** dim, 5), sentinel)
    s = eb.Solver(dim, order)
    g_luh, g_lim = dev(luh), dev(lim0)
    s.project_on_fv_limiter_space(g_luh, g_lim, n)
    got = host(g_lim)
    exp = np.stack([k.project_fv(luh[c], lim0[c]).reshape(E ** dim, 5) for c in range(n)])
    assert rel(got, exp) < RTOL
    assert np.array_equal(got == sentinel, exp == sentinel)  # ghost layers untouched
    lim = states(rng, (n, E ** dim))
    g_lim = dev(lim)
    g_out = dev(np.zeros_like(luh))
    s.project_on_dg_space(g_lim, g_out, n)
    exp = np.stack([k.project_dg(lim[c]).reshape(-1, 5) for c in range(n)])
    assert rel(host(g_out), exp) < RTOL


@pytest.mark.parametrize("dim,order,n", [(2, 3, 40), (2, 5, 33), (3, 3, 12), (3, 5, 7)])
def test_musclhancock_update_vs_oracle(eb, dim, order, n):
    rng = np.random.default_rng(100 * dim + order)
    k = pyoracle.Kernels(dim, order)
    E = 2 * order + 5
    lim = states(rng, (n, E ** dim))
    dx = [0.05, 0.04, 0.045][:dim]
    dt = 2e-4
    cells = rng.permutation(n)[: (2 * n) // 3].astype(np.int32)  # a ragged subset, shuffled
    s = eb.Solver(dim, order)
    g_lim, g_old = dev(lim), dev(np.zeros_like(lim))
    g_luh = dev(np.zeros((n, (order + 1) ** dim, 5)))
    g_list = dev(cells, torch.int32)
    g_dt = dev(np.array([dt]))
    nb = s.fv_musclhancock_scratch_bytes(len(cells))
    assert (nb == 0) == (dim == 2)
    scratch = torch.empty(max(nb, 8) // 8, dtype=torch.float64, device="cuda")
    s.fv_musclhancock_update(g_lim, g_old, g_luh, g_dt, dx, len(cells), g_list, scratch, nb)
    got, old, luh = host(g_lim), host(g_old), host(g_luh)
    for c in range(n):
        if c in set(cells.tolist()):
            exp = k.musclhancock(lim[c], dx, dt).reshape(E ** dim, 5)
            assert rel(got[c], exp) < RTOL, c
            assert np.array_equal(old[c], lim[c])
            assert rel(luh[c], k.project_dg(got[c]).reshape(-1, 5)) < RTOL
        else:
            assert np.array_equal(got[c], lim[c]) and not old[c].any() and not luh[c].any()


def test_musclhancock_scratch_limits(eb):
    """3D needs scratch: less than one block's share is refused on the host;
    room for a single block gives the same result as the full grid"""
    rng = np.random.default_rng(5)
    dim, order, n = 3, 3, 9
    E = 2 * order + 5
    lim = states(rng, (n, E ** dim))
    s = eb.Solver(dim, order)
    g_dt = dev(np.array([1e-4]))
    dx = [0.05, 0.05, 0.05]
    full = s.fv_musclhancock_scratch_bytes(n)
    outs = []
    for nbytes in (full, None):
        g_lim, g_old = dev(lim), dev(np.zeros_like(lim))
        if nbytes is None:  # room for exactly one block: the grid-stride loop does all cells
            one = s.fv_musclhancock_scratch_bytes(1)
            scratch = torch.empty(one // 8, dtype=torch.float64, device="cuda")
            s.fv_musclhancock_update(g_lim, g_old, None, g_dt, dx, n, None, scratch, one)
        else:
            scratch = torch.empty(nbytes // 8, dtype=torch.float64, device="cuda")
            s.fv_musclhancock_update(g_lim, g_old, None, g_dt, dx, n, None, scratch, nbytes)
        outs.append(host(g_lim))
    assert np.array_equal(outs[0], outs[1])
    with pytest.raises(eb.ExaError, match="scratch"):
        s.fv_musclhancock_update(dev(lim), dev(np.zeros_like(lim)), None, g_dt, dx, n, None,
                                 torch.empty(1, dtype=torch.float64, device="cuda"), 8)
