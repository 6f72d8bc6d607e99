"""The oracle's AMR transfer operators (oracle/amr.c; the reference's
amrRoutines.cpph) and the plotters' equidistant vertex projection, pinned by
the reference's own property tests (GenericEulerKernelTest2D.cpp:1037-1190:
constants survive prolongation, the restrictions of all descendants of a
constant add up to it), by exactness on polynomials of degree N, and against
the reference's routines compiled from source (oracle/_ref)."""
import itertools

import numpy as np
import pytest

import pyoracle

needs_ref = pytest.mark.skipif(not (pyoracle.ref_available(2) and pyoracle.ref_available(3)),
                               reason="oracle/_ref not built")


def gl(N):
    return np.array(pyoracle.table("nodes", N))


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("levelDelta", [1, 2])
def test_constants_reference_property(dim, levelDelta):
    # testFaceUnknownsProjection / testVolumeUnknownsProjection: nVar 1, nPar 1, N 3;
    # the projector is stored with 13 digits, so its rows sum to 1 within ~1e-12
    N, nv, npar = 3, 1, 1
    b = N + 1
    subs = 3 ** levelDelta
    ones_v, ones_f, ones_ff = np.ones(b ** dim * 2), np.ones(b ** (dim - 1) * 2), np.ones(b ** (dim - 1))
    acc_v, acc_f, acc_ff = np.zeros_like(ones_v), np.zeros_like(ones_f), np.zeros_like(ones_ff)
    for idx in itertools.product(range(subs), repeat=dim):
        fv = pyoracle.amr("volume_prolongation", dim, N, nv, npar, levelDelta, idx, coarse=ones_v)
        np.testing.assert_allclose(fv, ones_v, rtol=0, atol=1e-10)
        acc_v = pyoracle.amr("volume_restriction", dim, N, nv, npar, levelDelta, idx, coarse=acc_v, fine=ones_v)
    np.testing.assert_allclose(acc_v, ones_v, rtol=0, atol=1e-10)
    for idx in itertools.product(range(subs), repeat=dim - 1):
        fq, ff = pyoracle.amr("face_prolongation", dim, N, nv, npar, levelDelta, idx, coarse=ones_f, coarse_flux=ones_ff)
        np.testing.assert_allclose(fq, ones_f, rtol=0, atol=1e-10)
        np.testing.assert_allclose(ff, ones_ff, rtol=0, atol=1e-10)
        acc_f, acc_ff = pyoracle.amr("face_restriction", dim, N, nv, npar, levelDelta, idx, coarse=acc_f,
                                     fine=ones_f, coarse_flux=acc_ff, fine_flux=ones_ff)
    np.testing.assert_allclose(acc_f, ones_f, rtol=0, atol=1e-10)
    np.testing.assert_allclose(acc_ff, ones_ff, rtol=0, atol=1e-10)


@pytest.mark.parametrize("dim,N,levelDelta", [(2, 3, 1), (2, 5, 2), (3, 3, 1), (3, 4, 2)])
def test_polynomials_prolongate_exactly_and_restrict_back(dim, N, levelDelta):
    """a polynomial of degree N sampled at the coarse nodes prolongates to its
    samples at the fine nodes; restricting all descendants returns it"""
    rng = np.random.default_rng(dim * 10 + N)
    x = gl(N)
    coef = rng.normal(size=(N + 1,) * dim)

    def sample(lo, h):  # nodes of the subcell [lo, lo + h] per axis, x fastest
        pts = [lo[k] + h * x for k in range(dim)]
        grids = np.meshgrid(*pts[::-1], indexing="ij")  # (z,) y, x
        val = np.zeros(grids[0].shape)
        for e in itertools.product(range(N + 1), repeat=dim):
            term = coef[e]
            for k in range(dim):
                term = term * grids[dim - 1 - k] ** e[k]
            val = val + term
        return val.reshape(-1, 1)

    coarse = sample([0.0] * dim, 1.0)
    subs = 3 ** levelDelta
    h = 1.0 / subs
    acc = np.zeros_like(coarse).ravel()
    for idx in itertools.product(range(subs), repeat=dim):
        fine = pyoracle.amr("volume_prolongation", dim, N, 1, 0, levelDelta, idx, coarse=coarse)
        want = sample([i * h for i in idx], h).ravel()
        np.testing.assert_allclose(fine, want, rtol=0, atol=1e-11 * np.max(np.abs(want)))
        acc = pyoracle.amr("volume_restriction", dim, N, 1, 0, levelDelta, idx, coarse=acc, fine=want)
    np.testing.assert_allclose(acc, coarse.ravel(), rtol=0, atol=1e-11 * np.max(np.abs(coarse)))


@needs_ref
@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("N,nv,npar", [(3, 5, 0), (5, 5, 0), (4, 9, 3), (3, 5, 1)])
@pytest.mark.parametrize("levelDelta", [1, 2, 3])
def test_amr_vs_reference(dim, N, nv, npar, levelDelta):
    rng = np.random.default_rng(dim * 1000 + N * 100 + nv * 10 + levelDelta)
    b, nd = N + 1, nv + npar
    subs = 3 ** levelDelta
    idx = [int(rng.integers(0, subs)) for _ in range(dim)]
    u, v = rng.normal(size=b ** dim * nd), rng.normal(size=b ** dim * nd)

    def close(a, r):
        assert np.max(np.abs(a - r)) <= 1e-13 * max(np.max(np.abs(r)), 1.0)

    close(pyoracle.amr("volume_prolongation", dim, N, nv, npar, levelDelta, idx, coarse=u),
          pyoracle.amr("volume_prolongation", dim, N, nv, npar, levelDelta, idx, coarse=u, impl="ref"))
    close(pyoracle.amr("volume_restriction", dim, N, nv, npar, levelDelta, idx, coarse=v, fine=u),
          pyoracle.amr("volume_restriction", dim, N, nv, npar, levelDelta, idx, coarse=v, fine=u, impl="ref"))
    fq, ff = rng.normal(size=b ** (dim - 1) * nd), rng.normal(size=b ** (dim - 1) * nv)
    cq, cf = rng.normal(size=b ** (dim - 1) * nd), rng.normal(size=b ** (dim - 1) * nv)
    a = pyoracle.amr("face_prolongation", dim, N, nv, npar, levelDelta, idx[:dim - 1], coarse=cq, coarse_flux=cf)
    r = pyoracle.amr("face_prolongation", dim, N, nv, npar, levelDelta, idx[:dim - 1], coarse=cq, coarse_flux=cf,
                     impl="ref")
    close(a[0], r[0])
    close(a[1], r[1])
    a = pyoracle.amr("face_restriction", dim, N, nv, npar, levelDelta, idx[:dim - 1], coarse=cq, fine=fq,
                     coarse_flux=cf, fine_flux=ff)
    r = pyoracle.amr("face_restriction", dim, N, nv, npar, levelDelta, idx[:dim - 1], coarse=cq, fine=fq,
                     coarse_flux=cf, fine_flux=ff, impl="ref")
    close(a[0], r[0])
    close(a[1], r[1])


@needs_ref
@pytest.mark.parametrize("dim,N", [(2, 3), (2, 5), (3, 3), (3, 5)])
def test_plot_vertices_vs_reference(dim, N):
    rng = np.random.default_rng(dim + N)
    u = rng.normal(size=(N + 1) ** dim * 5)
    a = pyoracle.plot_vertices(dim, N, 5, u)
    r = pyoracle.plot_vertices(dim, N, 5, u, impl="ref")
    assert np.max(np.abs(a - r)) <= 1e-13 * np.max(np.abs(r))
    # the corner vertex of a constant is the constant (GenericEulerKernelTest.cpp:67-121)
    one = pyoracle.plot_vertices(dim, N, 1, np.ones((N + 1) ** dim))
    np.testing.assert_allclose(one, 1.0, rtol=0, atol=1e-10)
