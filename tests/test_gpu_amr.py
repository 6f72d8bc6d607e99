"""GPU parity of the AMR transfer operators (exa_volume/face_unknowns_*),
the plotters' vertex projection (exa_plot_vertices) and the VTK writer
(exa_mesh_write_vtk) against the oracle (oracle/amr.c), through the C ABI.

Bar: 1e-12 relative (max-norm) per transfer; the GPU applies the tensor
products one axis at a time where the reference sums the full product, so
results agree to rounding. Restrictions of several descendants into one
ancestor are summed with atomics (order not fixed), also 1e-12.
"""
import itertools
import os
import struct

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


def ints(a):
    return dev(np.asarray(a, dtype=np.int32), torch.int32)


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


CASES = [(2, 3, 0), (2, 5, 0), (3, 3, 0), (3, 5, 0), (3, 4, 2), (2, 5, 1)]  # (dim, N, pde)
SHAPE = {0: (5, 0), 1: (5, 1), 2: (9, 3)}


@pytest.mark.parametrize("dim,N,pde", CASES)
def test_volume_transfers_vs_oracle(eb, dim, N, pde):
    rng = np.random.default_rng(dim * 100 + N * 10 + pde)
    nv, npar = SHAPE[pde]
    nd, P = nv + npar, (N + 1) ** dim
    s = eb.Solver(dim, N, pde)
    ncoarse, nfine = 5, 24
    coarse = rng.normal(size=(ncoarse, P * nd))
    ld = rng.integers(1, 4, size=nfine).astype(np.int32)
    idx = np.zeros((nfine, 3), dtype=np.int32)
    for k in range(nfine):
        idx[k, :dim] = rng.integers(0, 3 ** ld[k], size=dim)
    par = rng.integers(0, ncoarse, size=nfine).astype(np.int32)
    fine_ids = rng.permutation(nfine).astype(np.int32)
    fine = dev(np.full((nfine, P * nd), 7.0))
    s.volume_unknowns_prolongation(fine, dev(coarse), nfine, ints(fine_ids), ints(par), ints(ld), ints(idx))
    got = host(fine)
    for k in range(nfine):
        want = pyoracle.amr("volume_prolongation", dim, N, nv, npar, int(ld[k]), idx[k, :dim], coarse=coarse[par[k]])
        assert rel(got[fine_ids[k]], want) < RTOL
    # restriction: random fine data added into the coarse cells (several per ancestor)
    fdat = rng.normal(size=(nfine, P * nd))
    acc = dev(coarse.copy())
    s.volume_unknowns_restriction(acc, dev(fdat), nfine, ints(fine_ids), ints(par), ints(ld), ints(idx))
    want = coarse.copy()
    for k in range(nfine):
        want[par[k]] = pyoracle.amr("volume_restriction", dim, N, nv, npar, int(ld[k]), idx[k, :dim],
                                    coarse=want[par[k]], fine=fdat[fine_ids[k]])
    assert rel(host(acc), want) < RTOL


@pytest.mark.parametrize("dim,N,pde", CASES)
def test_face_transfers_vs_oracle(eb, dim, N, pde):
    rng = np.random.default_rng(dim * 100 + N * 10 + pde + 7)
    nv, npar = SHAPE[pde]
    nd, F = nv + npar, (N + 1) ** (dim - 1)
    s = eb.Solver(dim, N, pde)
    nslots, nt = 12, 20
    q, f = rng.normal(size=(nslots, F * nd)), rng.normal(size=(nslots, F * nv))
    ld = rng.integers(1, 4, size=nt).astype(np.int32)
    idx = np.zeros((nt, 2), dtype=np.int32)
    for k in range(nt):
        idx[k, :dim - 1] = rng.integers(0, 3 ** ld[k], size=dim - 1)
    src = rng.integers(0, nslots, size=nt).astype(np.int32)
    dst = rng.permutation(nt).astype(np.int32)
    qf, ff = dev(np.zeros((nt, F * nd))), dev(np.zeros((nt, F * nv)))
    s.face_unknowns_prolongation(qf, ff, dev(q), dev(f), nt, ints(dst), ints(src), ints(ld), ints(idx))
    gq, gf = host(qf), host(ff)
    for k in range(nt):
        wq, wf = pyoracle.amr("face_prolongation", dim, N, nv, npar, int(ld[k]), idx[k, :dim - 1], coarse=q[src[k]],
                              coarse_flux=f[src[k]])
        assert rel(gq[dst[k]], wq) < RTOL and rel(gf[dst[k]], wf) < RTOL
    fq, fff = rng.normal(size=(nt, F * nd)), rng.normal(size=(nt, F * nv))
    aq, af = dev(q.copy()), dev(f.copy())
    s.face_unknowns_restriction(aq, af, dev(fq), dev(fff), nt, ints(dst), ints(src), ints(ld), ints(idx))
    wq, wf = q.copy(), f.copy()
    for k in range(nt):
        wq[src[k]], wf[src[k]] = pyoracle.amr("face_restriction", dim, N, nv, npar, int(ld[k]), idx[k, :dim - 1],
                                              coarse=wq[src[k]], fine=fq[dst[k]], coarse_flux=wf[src[k]],
                                              fine_flux=fff[dst[k]])
    assert rel(host(aq), wq) < RTOL and rel(host(af), wf) < RTOL


def test_invalid_transfers_are_skipped(eb):
    s = eb.Solver(2, 3, 0)
    P = 16 * 5
    fine = dev(np.full((3, P), 7.0))
    coarse = dev(np.ones((1, P)))
    # level 0, level 13, index 9 at level 2 (>= 3^2): all skipped, nothing written
    s.volume_unknowns_prolongation(fine, coarse, 3, ints([0, 1, 2]), ints([0, 0, 0]), ints([0, 13, 2]),
                                   ints([[0, 0, 0], [0, 0, 0], [9, 0, 0]]))
    assert np.all(host(fine) == 7.0)


@pytest.mark.parametrize("dim,N,pde", [(2, 3, 0), (3, 5, 0), (3, 4, 2)])
def test_plot_vertices_vs_oracle(eb, dim, N, pde):
    rng = np.random.default_rng(dim + N + pde)
    nd = sum(SHAPE[pde])
    P = (N + 1) ** dim
    s = eb.Solver(dim, N, pde)
    u = rng.normal(size=(9, P * nd))
    out = dev(np.zeros((9, P * nd)))
    s.plot_vertices(dev(u), out, 9)
    got = host(out)
    for c in range(9):
        assert rel(got[c], pyoracle.plot_vertices(dim, N, nd, u[c])) < RTOL


def read_vtk(path):
    """minimal legacy-VTK reader for what exa_mesh_write_vtk writes"""
    data = open(path, "rb").read()
    lines = data.split(b"\n")
    binary = lines[2].strip() == b"BINARY"
    pos = sum(len(l) + 1 for l in lines[:4])
    out = {}

    def header():
        nonlocal pos
        end = data.index(b"\n", pos)
        h = data[pos:end].decode().split()
        pos = end + 1
        return h

    def values(count, kind):
        nonlocal pos
        if binary:
            fmt, size = (">d", 8) if kind == "d" else (">i", 4)
            vals = np.array(struct.unpack(">" + fmt[1] * count, data[pos:pos + size * count]))
            pos += size * count + 1
            return vals
        toks = []
        while len(toks) < count:
            end = data.index(b"\n", pos)
            toks.extend(data[pos:end].split())
            pos = end + 1
        return np.array([float(t) for t in toks]) if kind == "d" else np.array([int(t) for t in toks])

    h = header()
    npts = int(h[1])
    out["points"] = values(3 * npts, "d").reshape(npts, 3)
    h = header()
    out["cells"] = values(int(h[2]), "i")
    h = header()
    out["types"] = values(int(h[1]), "i")
    header()
    h = header()
    nq = int(h[3])
    header()
    out["Q"] = values(npts * nq, "d").reshape(npts, nq)
    header()
    header()
    out["time"] = values(npts, "d")
    if pos < len(data):  # further vertex scalars (one value each)
        name = header()[1]
        header()
        out[name] = values(npts, "d")
    return out


@pytest.mark.parametrize("dim,N,cells", [(2, 3, (3, 2)), (3, 3, (2, 2, 1))])
def test_write_vtk(eb, tmp_path, dim, N, cells):
    from exahype_b200 import problems
    s = eb.Solver(dim, N, eb.PDE_EULER)
    m = eb.Mesh(s, cells, [0.5] * dim, [1.5] * dim, eb.BC_PERIODIC)
    u = problems.gaussian_pulse_2d(N, cells, seed=1)[0] if dim == 2 else problems.gaussian_pulses_3d(N, cells, seed=1)[0]
    m.set_solution(u)
    m.init(0.0)
    m.step(2)
    sol = m.get_solution()
    b, n = N + 1, int(np.prod(cells))
    ref_q = np.concatenate([pyoracle.plot_vertices(dim, N, 5, sol[c]).reshape(-1, 5) for c in range(n)])
    t = m.state()["t"]
    res = []
    for binary in (False, True):
        path = str(tmp_path / ("m%d.vtk" % binary))
        m.write_vtk(path, binary=binary)
        v = read_vtk(path)
        assert v["points"].shape == (n * b ** dim, 3)
        assert rel(v["Q"], ref_q) < RTOL
        assert np.all(v["time"] == t)
        sub = N ** dim
        assert len(v["types"]) == n * sub and np.all(v["types"] == (11 if dim == 3 else 8))
        assert len(v["cells"]) == n * sub * (1 + 2 ** dim)
        # vertex coordinates: offset + (cell + i / N) * dx
        dx = 1.5 / np.array(cells)
        lo = v["points"].min(axis=0)[:dim]
        hi = v["points"].max(axis=0)[:dim]
        assert np.allclose(lo, 0.5) and np.allclose(hi, 0.5 + 1.5)
        res.append(v)
    assert np.array_equal(res[0]["cells"], res[1]["cells"])
    assert np.array_equal(res[0]["points"], res[1]["points"])  # text uses 17 digits: round-trips exactly
    assert np.array_equal(res[0]["Q"], res[1]["Q"])


@pytest.mark.parametrize("dim,N,cells", [(2, 3, (4, 5)), (3, 5, (2, 3, 2))])
def test_write_vtk_legendre(eb, tmp_path, dim, N, cells):
    """ADERDG2LegendreVTK layout: the points are every cell's Gauss-Legendre
    nodes and the values the nodal solution itself, text and binary alike"""
    from exahype_b200 import problems
    s = eb.Solver(dim, N, eb.PDE_EULER)
    m = eb.Mesh(s, cells, [0.5] * dim, [1.5] * dim, eb.BC_PERIODIC)
    u = problems.gaussian_pulse_2d(N, cells, seed=1)[0] if dim == 2 else problems.gaussian_pulses_3d(N, cells, seed=1)[0]
    m.set_solution(u)
    m.init(0.0)
    m.step(2)
    sol = m.get_solution()
    X = problems.node_coordinates(dim, N, cells, offset=(0.5, 0.5, 0.5), size=(1.5, 1.5, 1.5)).reshape(-1, dim)
    res = []
    for binary in (False, True):
        path = str(tmp_path / ("l%d.vtk" % binary))
        m.write_vtk_legendre(path, binary=binary)
        v = read_vtk(path)
        assert np.array_equal(v["Q"], sol.reshape(-1, 5))
        assert np.allclose(v["points"][:, :dim], X, rtol=0, atol=1e-14)
        assert len(v["types"]) == int(np.prod(cells)) * N ** dim
        res.append(v)
    assert np.array_equal(res[0]["points"], res[1]["points"])


def test_lmesh_write_vtk(eb, tmp_path):
    """LimitingADERDG2CartesianVTK layout: the projected DG solution of a
    limiting mesh and every vertex's cell limiter status"""
    from exahype_b200 import problems
    N, cells = 3, (10, 10)
    s = eb.Solver(2, N, eb.PDE_EULER)
    lu, fv, _ = problems.explosion(2, N, cells, seed=0)
    g = eb.LimitingMesh(s, cells, [0.0, 0.0], [1.0, 1.0], eb.BC_OUTFLOW)
    g.set_solution(lu)
    g.set_fv_initial(fv)
    g.init(0.0)
    g.step(3)
    sol, st = g.get_solution(), g.status()
    assert (st > 0).any()
    b, n = N + 1, cells[0] * cells[1]
    ref_q = np.concatenate([pyoracle.plot_vertices(2, N, 5, sol[c]).reshape(-1, 5) for c in range(n)])
    for binary in (False, True):
        path = str(tmp_path / ("lm%d.vtk" % binary))
        g.write_vtk(path, binary=binary)
        v = read_vtk(path)
        assert rel(v["Q"], ref_q) < RTOL
        assert np.array_equal(v["Limiter-Status"], np.repeat(st, b * b).astype(np.float64))
