"""The FP64 slow-term table of the force kernel's precise pass (host-only):
its polynomials against the slow pair energy written from scipy's FP64 erf,
and their derivatives against the slow force factor."""
import math

import numpy as np
import pytest
from scipy.special import erf, erfc

import nbk
from helpers import PARAMS


DEG = 5    # polynomial degree of a row (6 coefficients)


def _eval(T, step, s):
    k = np.rint(s / step).astype(int)
    w = s - step * k
    c = T[k]
    p = c[:, DEG].copy()
    dp = np.zeros_like(p)
    for n in range(DEG - 1, -1, -1):
        dp = dp * w + p
        p = p * w + c[:, n]
    return p, dp


# (ewaldcof, cutoff, pairlistdist): the benchmark's, the Ewald coefficients
# that PME tolerance 1e-6 gives for 10 and 8 A cutoffs, a long and a short one
@pytest.mark.parametrize("beta,cutoff,pl", [(PARAMS.ewaldcof, PARAMS.cutoff, PARAMS.pairlistdist),
                                            (0.34, 10.0, 11.5), (0.43, 8.0, 9.5), (0.2, 14.0, 16.0),
                                            (0.6, 6.0, 7.5)])
def test_slow_table_matches_the_slow_term(beta, cutoff, pl):
    T, step = nbk.slow_table(beta, cutoff, pl)
    assert T.shape[1] == DEG + 1
    assert step <= 32.0 and math.log2(step) == round(math.log2(step))
    # rows cover s up to pairlistdist^2 + 2
    assert step * (T.shape[0] - 1) + step / 2 >= pl * pl + 2
    s = np.linspace(1.0, pl * pl, 200001)
    r = np.sqrt(s)
    rc = cutoff
    # E_slow per unit qq as the oracle writes it, h + (erfc(beta r) - 1)/r,
    # and the force factor (dE/dr)/r per unit qq,
    # -rc^-3 - (erfc - 1)/r^3 - (2 beta/sqrt(pi)) exp(-beta^2 r^2)/r^2
    h = (3.0 - s / rc ** 2) / (2.0 * rc)
    phi = h + (erfc(beta * r) - 1.0) / r
    g = (-1.0 / rc ** 3 + erf(beta * r) / r ** 3
         - 2.0 * beta / math.sqrt(math.pi) * np.exp(-beta * beta * s) / s)
    p, dp = _eval(T, step, s)
    # the builder's bound: 1e-12 of max |phi_s| + 1/rc
    assert np.abs(p - phi).max() <= 1e-12 * (np.abs(phi).max() + 1.0 / rc)
    # the derivative, one order less smooth, within 2e-9 of the largest factor
    assert np.abs(2.0 * dp - g).max() <= 2e-9 * np.abs(g).max()


def test_slow_table_rejects_bad_parameters():
    L = nbk.dev_lib()
    assert L.nbk_slow_table(0.26, -1.0, 13.5, None, 0, None) < 0
    assert L.nbk_slow_table(0.26, 12.0, 11.0, None, 0, None) < 0
    rows = L.nbk_slow_table(0.26, 12.0, 13.5, None, 0, None)
    out = np.zeros((rows - 1, DEG + 1))
    assert L.nbk_slow_table(0.26, 12.0, 13.5, out.ctypes.data, rows - 1, None) < 0
