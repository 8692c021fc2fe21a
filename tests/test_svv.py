"""Spectral vanishing viscosity operators (src/svv.cpp) on the CPU: the
library's SVV derivative and Fourier-mode factors against the oracle's
restatement, and the defining property of the filter."""
import numpy as np
import pytest

import semtex_oracle as O
import semtex_b200 as S


@pytest.mark.parametrize("np_,mn,eps", [(6, 3, 0.05), (9, 4, 0.1), (11, 5, 0.02), (13, 0, 0.3)])
def test_svv_derivative_matches_oracle(np_, mn, eps):
    D, Z = S.svv(np_, eps, mn, 16, 0.02, 2, 0.01)
    z, w, D0 = O.gll(np_)
    Do = O.svv_derivative(z, w, D0, eps, mn, 0.01)
    assert np.abs(D - Do).max() < 1e-12 * max(1.0, np.abs(Do).max())
    assert np.abs(D - D0).max() > 1e-3                      # the filter acts
    np.testing.assert_allclose(Z, O.svv_z(16, 8, 0.02, 2, 0.01), rtol=0, atol=1e-15)


@pytest.mark.parametrize("np_,mn", [(7, 3), (10, 5)])
def test_svv_keeps_modes_up_to_mn(np_, mn):
    # S_k = 1 for k <= mN: the SVV derivative of a polynomial of degree <= mN
    # is its derivative; of degree N it is not
    D, _ = S.svv(np_, 0.1, mn, 1, 0.0, -1, 0.01)
    z, _, D0 = O.gll(np_)
    for d in range(mn + 1):
        np.testing.assert_allclose(D @ z ** d, D0 @ z ** d, rtol=0, atol=1e-10)
    assert np.abs(D @ z ** (np_ - 1) - D0 @ z ** (np_ - 1)).max() > 1e-3


@pytest.mark.parametrize("eps,mn", [(0.0, 3), (0.1, -1), (0.1, 8)])
def test_svv_off_is_the_plain_derivative(eps, mn):
    D, Z = S.svv(9, eps, mn, 8, eps, mn, 0.01)
    np.testing.assert_allclose(D, O.gll(9)[2], rtol=0, atol=1e-13)
    np.testing.assert_array_equal(Z, np.ones(4))
