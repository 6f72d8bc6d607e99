"""exa_fv_musclhancock_update_noalloc (library-owned static scratch, no device
allocation) against exa_fv_musclhancock_update (caller scratch): two calls in a
row, each fed the previous call's output, must agree bit for bit -- both run
the same per-cell computation, only the scratch and the grid size differ.

The 32 MiB static array holds the scratch of 151 blocks for 3D N=3 and of 47
for 3D N=5; the larger cases list more cells than that, so the static path's
blocks loop over several cells each and reuse their slice of the array."""
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


def states(rng, shape):
    q = np.zeros(shape + (5,))
    q[..., 0] = 1.0 + 0.3 * rng.random(shape)
    q[..., 1:4] = 0.2 * (rng.random(shape + (3,)) - 0.5)
    q[..., 4] = 2.5 + 0.5 * rng.random(shape)
    return q


STATIC_BYTES = 32 << 20


@pytest.mark.parametrize("dim,order,n,beyond_cap", [(3, 3, 200, False), (3, 5, 60, False), (2, 5, 150, False),
                                                    (3, 5, 200, True), (3, 3, 800, True)])
def test_noalloc_matches_caller_scratch_two_calls(eb, dim, order, n, beyond_cap):
    rng = np.random.default_rng(7 * dim + order)
    E = 2 * order + 5
    lim0 = torch.as_tensor(states(rng, (n, E ** dim))).cuda()
    dx = [0.05, 0.04, 0.045][:dim]
    dt = torch.tensor([2e-4], dtype=torch.float64, device="cuda")
    cells = torch.as_tensor(rng.permutation(n)[: (3 * n) // 4].astype(np.int32)).cuda()
    m = int(cells.numel())
    s = eb.Solver(dim, order)
    nb = s.fv_musclhancock_scratch_bytes(m)
    if beyond_cap:
        per_block = s.fv_musclhancock_scratch_bytes(1)
        assert m > STATIC_BYTES // per_block, "this case must list more cells than the static array's blocks"
    scratch = torch.empty(max(nb, 8) // 8, dtype=torch.float64, device="cuda")

    a_lim, a_old = lim0.clone(), torch.zeros_like(lim0)
    b_lim, b_old = lim0.clone(), torch.zeros_like(lim0)
    a_luh = torch.zeros((n, (order + 1) ** dim, 5), dtype=torch.float64, device="cuda")
    b_luh = torch.zeros_like(a_luh)
    for call in range(2):
        s.fv_musclhancock_update(a_lim, a_old, a_luh, dt, dx, m, cells, scratch, nb)
        s.fv_musclhancock_update_noalloc(b_lim, b_old, b_luh, dt, dx, m, cells)
        torch.cuda.synchronize()
        assert torch.equal(a_lim, b_lim), "call %d: patches differ" % call
        assert torch.equal(a_old, b_old), "call %d: previous patches differ" % call
        assert torch.equal(a_luh, b_luh), "call %d: DG projections differ" % call
    assert not torch.equal(a_lim, lim0)  # the patches did change
