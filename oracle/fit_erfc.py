"""Least-squares fit of the erfc approximation used by the force kernels.

Form (Hastings' rational approximation, the form of Abramowitz & Stegun
7.1.26):   erfc(x) = t * P(t) * exp(-x^2),  t = 1 / (1 + p x),  x in [0, 4]
with P a polynomial of degree 7. p and the coefficients are fitted here by
weighted least squares on the relative error (exact erfc from scipy); the
printed constants are the ones in namd-3.0_b200/csrc/nbk_internal.cuh (kept
here beside the oracle as their provenance). Max relative error of
the fit: 1.6e-8, below FP32 resolution. The kernels share exp(-x^2) between
erfc and the force's Gaussian term, so erfc costs one reciprocal and 8 FMAs.

    python fit_erfc.py
"""
import numpy as np
from scipy.optimize import minimize_scalar
from scipy.special import erfc

X = np.linspace(0.0, 4.0, 20001)
NTERMS = 8


def fit(p):
    t = 1.0 / (1.0 + p * X)
    y = erfc(X) * np.exp(X * X) / t
    V = np.vander(t, NTERMS, increasing=True)
    w = 1.0 / y
    c, *_ = np.linalg.lstsq(V * w[:, None], y * w, rcond=None)
    return c, np.abs((V @ c - y) / y).max()


def main():
    best = minimize_scalar(lambda p: fit(p)[1], bounds=(0.2, 0.8), method="bounded",
                           options={"xatol": 1e-10})
    p = best.x
    c, err = fit(p)
    print(f"// max relative error {err:.3e}")
    print(f"constexpr float kErfcP = {p:.9e}f;")
    print("constexpr float kErfcC[8] = {" + ", ".join(f"{v:.9e}f" for v in c) + "};")


if __name__ == "__main__":
    main()
