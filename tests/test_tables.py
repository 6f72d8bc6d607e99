"""The generated DG operator tables (exahype_b200/csrc/gen_tables.py, computed
from first principles) against the reference's own tables, dumped by its init
code (kernels/DGMatrices.cpp, GaussLegendreQuadrature.cpp,
LimiterProjectionMatrices.cpp) into tests/golden/ref_tables.npz."""
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(REPO, "exahype_b200", "csrc"))
import gen_tables  # noqa: E402

REF = np.load(os.path.join(REPO, "tests", "golden", "ref_tables.npz"))


@pytest.mark.parametrize("N", [3, 5])
def test_13_digit_operators_bit_identical(N):
    """Kxi, iK1, dudx, FCoeff and fineGridProjector1d are stored by the reference with 13
    significant digits; rounding the exact operators the same way reproduces
    them bit for bit for the orders the workloads use."""
    t = gen_tables.build(N)
    for name in ("Kxi", "iK1", "dudx", "FCoeff", "fineGridProjector1d"):
        assert np.array_equal(np.array(t[name]), REF["%s/%d" % (name, N)]), name


@pytest.mark.parametrize("N", range(1, 10))
def test_all_tables_close(N):
    t = gen_tables.build(N)
    for name in gen_tables.NAMES:
        ref = REF["%s/%d" % (name, N)]
        mine = np.array(t[name])
        assert mine.shape == ref.shape, name
        # the reference's 16-digit quadrature/extrapolation values carry ~1e-15
        # of numerical error; 13-digit tables may differ in the last digit
        atol = 2e-13 if name in ("Kxi", "iK1", "dudx", "FCoeff", "fineGridProjector1d",
                                 "equidistantGridProjector1d") else 1e-14
        np.testing.assert_allclose(mine, ref, rtol=3e-12, atol=atol, err_msg=name)


def test_quadrature_identities():
    for N in range(1, 10):
        t = gen_tables.build(N)
        w, x = np.array(t["weights"]), np.array(t["nodes"])
        assert abs(w.sum() - 1) < 1e-15
        for k in range(2 * N + 2):  # b-point Gauss is exact to degree 2N+1
            assert abs(np.sum(w * x ** k) - 1.0 / (k + 1)) < 1e-14
        # Kxi + Kxi^T = FR FR^T - FL FL^T (summation by parts)
        K = np.array(t["Kxi"]).reshape(N + 1, N + 1)
        FL, FR = np.array(t["FLCoeff"]), np.array(t["FRCoeff"])
        assert np.max(np.abs(K + K.T - (np.outer(FR, FR) - np.outer(FL, FL)))) < 1e-11
