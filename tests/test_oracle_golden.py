"""Pins the FP64 oracle's pair formulas to the reference's own pair-math code.

tests/golden/ref_pairmath.npz holds outputs of the reference's device
functions cudaNBForceMagCalc_VdwEnergySwitch_PMEC1 and
cudaModExclForceMagCalc_VdwEnergySwitch_PMEC1
(src/CudaComputeNonbondedInteractions.h:190-254), compiled host-side from the
reference tree (oracle/ref_pin) by tests/golden/make_golden.py. The reference
evaluates in FP32, so agreement is to FP32 noise: every column within 5e-5 of
its RMS, and the median relative error within 1e-5. A wrong sign, factor or
term would show as an O(1) difference.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))


def _oracle_pairs(fn, r2, qq, A, B, consts):
    n = len(r2)
    out = np.zeros((n, 5))
    dp = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    ins = [dp(r2), dp(qq), dp(A), dp(B)]
    fn.argtypes = [C.c_int] + [C.c_void_p] * 4 + [C.c_double] * 3 + [C.c_void_p]
    fn(n, *[a.ctypes.data for a in ins], *map(float, consts), out.ctypes.data)
    return out


@pytest.mark.parametrize("kind", ["nonbonded", "modified"])
def test_oracle_matches_reference_pair_math(kind):
    g = np.load(os.path.join(HERE, "golden", "ref_pairmath.npz"))
    L = oracle.lib()
    if kind == "nonbonded":
        out = _oracle_pairs(L.oracle_pair_nonbonded, g["r2"], g["qq"], g["A"], g["B"], g["consts"])
        ref = g["out_nb"].astype(np.float64)
    else:
        out = _oracle_pairs(L.oracle_pair_modified, g["r2"], g["qq"], g["dA"], g["dB"], g["consts"])
        # the bonded kernel applies F_i += f (x_i - x_j): opposite force sign
        out[:, :2] *= -1.0
        ref = g["out_mod"].astype(np.float64)
    for k in range(5):
        rms = np.sqrt(np.mean(out[:, k] ** 2))
        if rms == 0:
            assert np.all(ref[:, k] == 0)
            continue
        d = np.abs(ref[:, k] - out[:, k])
        assert d.max() <= 5e-5 * rms, (kind, k, d.max() / rms)
        big = np.abs(out[:, k]) > 1e-3 * rms
        assert np.median(d[big] / np.abs(out[big, k])) <= 1e-5, (kind, k)


def test_oracle_force_is_energy_gradient():
    """g = (dE/dr)/r for every term, by central differences in FP64."""
    L = oracle.lib()
    r = np.linspace(1.2, 11.9, 400)
    h = 1e-6
    qq = np.full_like(r, 57.7)
    A = np.full_like(r, 4.0 * 0.15 * 3.15 ** 12)
    B = np.full_like(r, 4.0 * 0.15 * 3.15 ** 6)
    c = (12.0, 10.0, 0.2579)
    for fn in (L.oracle_pair_nonbonded, L.oracle_pair_modified):
        o = _oracle_pairs(fn, r * r, qq, A, B, c)
        op = _oracle_pairs(fn, (r + h) ** 2, qq, A, B, c)
        om = _oracle_pairs(fn, (r - h) ** 2, qq, A, B, c)
        # fast force = LJ + fast elec (energy columns 2, 3); slow = column 4
        dEf = ((op[:, 2] + op[:, 3]) - (om[:, 2] + om[:, 3])) / (2 * h) / r
        dEs = (op[:, 4] - om[:, 4]) / (2 * h) / r
        np.testing.assert_allclose(o[:, 0], dEf, rtol=1e-6, atol=1e-7 * np.abs(o[:, 0]).max())
        np.testing.assert_allclose(o[:, 1], dEs, rtol=1e-6, atol=1e-7 * np.abs(o[:, 1]).max())
