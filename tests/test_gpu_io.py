"""exa_mesh_step_io: streamed host input/output around every step gives the
same results, bit for bit, as uploading, stepping and downloading one step
at a time (the copies of neighbouring steps overlap, their order does not
change)."""
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


@pytest.mark.parametrize("nin,nout", [(1, 1), (3, 4)])
def test_step_io_matches_serial(eb, nin, nout):
    from exahype_b200 import problems
    dim, N, cells = 3, 3, (6, 6, 6)
    u, _ = problems.gaussian_pulses_3d(N, cells, seed=4)
    s = eb.Solver(dim, N)
    rng = np.random.default_rng(1)
    inputs = [u * (1.0 + 0.01 * rng.random(u.shape)) for _ in range(nin)]
    nbytes = u.size * 8
    steps = 7
    res = []
    for mode in ("io", "serial"):
        m = eb.Mesh(s, cells, [0.0] * dim, [1.0] * dim, eb.BC_PERIODIC)
        m.set_solution(u)
        m.init(0.0)
        pin_in = torch.empty(nin * u.size, dtype=torch.float64, pin_memory=True)
        pin_in.numpy().reshape(nin, -1)[:] = np.stack([x.reshape(-1) for x in inputs])
        pin_out = torch.zeros(nout * u.size, dtype=torch.float64, pin_memory=True)
        if mode == "io":
            m.step_io(pin_in.data_ptr(), nin, pin_out.data_ptr(), nout, nbytes, steps)
        else:
            for k in range(steps):
                m.upload_solution_async(pin_in.data_ptr() + (k % nin) * nbytes, nbytes)
                m.step(1)
                m.download_solution_async(pin_out.data_ptr() + (k % nout) * nbytes, nbytes)
        m.synchronize()
        res.append((pin_out.numpy().copy(), m.get_solution(), m.state()))
    (oa, ua, sa), (ob, ub, sb) = res
    assert np.array_equal(oa, ob) and np.array_equal(ua, ub)
    assert sa == sb and sa["steps"] == steps
