"""The 0-D outlet model (:mod:`zvcfd_b200.lumped`) against the reference's own RCR
(``zvcfd/lumped.py:181-218``), through golden vectors the reference produced
(``tests/golden/make_golden.py lumped``): steady coefficients, and 40 steps of step
coefficients and committed pressures under a pulsatile outflow, trapezoidal and backward
Euler, with constant and tabulated venous pressure; and the variable-step BDF coefficients and
the Carreau-Yasuda law of the same module family (CPU)."""

import numpy as np
import pytest

from fixtures import load

PARAMS = [(1e8, 1e-9, 1e9, 0.0), (2.0, 0.1, 5.0, 1.0),
          (0.5e8, 2e-9, 0.8e9, [(0.0, 100.0), (0.4, 300.0), (0.8, 100.0)])]


@pytest.mark.parametrize("method", ["trapezoidal", "euler"])
@pytest.mark.parametrize("i", range(len(PARAMS)))
def test_rcr_matches_reference(i, method):
    from zvcfd_b200.lumped import RCR

    g = load("lumped")
    rp, c, rd, pv = PARAMS[i]
    m = RCR(rp=rp, c=c, rd=rd, pv=pv, method=method)
    np.testing.assert_allclose(m.steady_coefficients(0.0), g[f"rcr{i}_{method}_steady"],
                               rtol=1e-14)
    m.initialise(1e-6 if rp > 10 else 0.3, 0.0)
    ref = g[f"rcr{i}_{method}_steps"]
    for t, q, a, r, p in ref:
        np.testing.assert_allclose(m.coefficients(t, 0.013), (a, r), rtol=1e-13, atol=1e-300)
        np.testing.assert_allclose(m.advance(q, t, 0.013), p, rtol=1e-13)


def test_bdf_coefficients_and_carreau_yasuda_match_reference():
    """Variable-step BDF1/2 coefficients (``zvcfd/fv/reference.py:143-153``) and the
    Carreau-Yasuda law (``zvcfd/rheology.py:37-62``) equal the reference's values."""
    from zvcfd_b200.fluid import CarreauYasuda
    from zvcfd_b200.solver import bdf_coefficients

    g = load("lumped")
    cases = [("bdf1", 1e-3, None, 1), ("bdf2", 1e-3, None, 1), ("bdf2", 1e-3, 1e-3, 2),
             ("bdf2", 2e-3, 1e-3, 2), ("bdf2", 0.5e-3, 1.5e-3, 2)]
    np.testing.assert_array_equal(np.array([bdf_coefficients(*c) for c in cases]), g["bdf"])
    gamma = g["cy_gamma"]
    np.testing.assert_allclose(CarreauYasuda()(gamma), g["cy_blood"], rtol=1e-15)
    np.testing.assert_allclose(CarreauYasuda(0.1, 0.004, 1.5, 1.7, 0.4)(gamma), g["cy_other"],
                               rtol=1e-15)
