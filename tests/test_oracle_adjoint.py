"""The FP64 oracle's adjoint (the reference gradient the GPU adjoint is checked
against) agrees with central differences of the FP64 loss, with the steps of
the differentiation workload: 1e-4 A in positions, 1e-4 e in charges, 1e-5 in
LJ sigma and epsilon."""
import numpy as np
import pytest

import nbk
import oracle
from helpers import PARAMS, mixed_box

QSCALE = np.sqrt(332.0636)


@pytest.fixture(scope="module")
def setup():
    s = mixed_box(seed=31, natoms=4000)
    p = nbk.Packed(s)
    o = oracle.Oracle(p, PARAMS)
    rng = np.random.default_rng(5)
    n = p.atomStorageSize
    w = rng.standard_normal((n, 3))
    return s, p, o, w


def test_position_and_charge_gradients(setup):
    s, p, o, w = setup
    cot = (w, w, 0.1, 0.1, 0.1)
    L, gX, gQ, gA, gB = o.adjoint(*cot)
    rng = np.random.default_rng(9)
    slots = rng.choice(p.slotOfAtom, 24, replace=False)
    X = o.xyzq
    checked = 0
    for k in slots:
        if o.near_cutoff(k, 0.01):
            continue
        for c in range(3):
            x0 = X[k, c]
            X[k, c] = np.float32(x0 + 1e-4)
            xp = float(X[k, c])
            Lp = o.loss_local(k, *cot)
            X[k, c] = np.float32(x0 - 1e-4)
            xm = float(X[k, c])
            Lm = o.loss_local(k, *cot)
            X[k, c] = x0
            fd = (Lp - Lm) / (xp - xm)
            assert abs(fd - gX[k, c]) <= 1e-5 * max(1.0, abs(gX[k, c])) + 1e-4, (k, c, fd, gX[k, c])
        q0 = X[k, 3]
        h = np.float32(1e-4 * QSCALE)
        X[k, 3] = q0 + h
        qp = float(X[k, 3])
        Lp = o.loss_local(k, *cot)
        X[k, 3] = q0 - h
        qm = float(X[k, 3])
        Lm = o.loss_local(k, *cot)
        X[k, 3] = q0
        fd = (Lp - Lm) / (qp - qm)
        assert abs(fd - gQ[k]) <= 1e-5 * max(1.0, abs(gQ[k])) + 1e-4, (k, fd, gQ[k])
        checked += 1
    assert checked >= 15


def test_lj_parameter_gradients(setup):
    s, p, o, w = setup
    cot = (w, w, 0.1, 0.1, 0.1)
    L, gX, gQ, gA, gB = o.adjoint(*cot)
    a = s.arrays()
    sig, eps = a["sigma"].copy(), a["epsilon"].copy()
    gS, gE = nbk.lj_param_grad(sig, eps, gA, gB, PARAMS.scaling)
    host = nbk.host_lib()
    dim = len(sig)

    def loss_with(sig2, eps2):
        import ctypes as C
        A, B, A14, B14 = (np.zeros(dim * dim) for _ in range(4))
        dp = lambda v: v.ctypes.data_as(C.POINTER(C.c_double))
        host.nbk_lj_table(dim, dp(np.ascontiguousarray(sig2)), dp(np.ascontiguousarray(eps2)), 0,
                          dp(A), dp(B), dp(A14), dp(B14))
        o2 = oracle.Oracle(p, PARAMS, lj=(dim, A, B, A14, B14))
        return o2.adjoint(*cot, grads=False)

    for t in (0, 5, 17):   # solute types
        for arr, g, h in ((sig, gS, 1e-5), (eps, gE, 1e-5)):
            v0 = arr[t]
            arr[t] = v0 + h
            Lp = loss_with(sig, eps)
            arr[t] = v0 - h
            Lm = loss_with(sig, eps)
            arr[t] = v0
            fd = (Lp - Lm) / (2 * h)
            assert abs(fd - g[t]) <= 1e-4 * max(1.0, abs(g[t])), (t, fd, g[t])
