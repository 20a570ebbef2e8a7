"""The adjoint behind a torch.autograd.Function (needs a B200).

The Function's forward is nbk_nonbonded_force (fast forces, slow forces and
the three energies, all summed exactly in fixed point or FP64), its backward
nbk_adjoint with the cotangents torch hands it; the wrapper lives only here,
in the tests. On the 24,000-atom mixed system of the differentiation workload
the gradient that torch.autograd.grad returns for

    L = sum w.F + sum w.Fslow + 0.1 (E_vdw + E_elec + E_slow),  w ~ N(0, 1),

is checked against the FP64 oracle's analytic gradient, and against central
differences of the product's own forward: steps of 1e-4 A in positions,
1e-4 e in charges and 1e-5 in the LJ sigma and epsilon of solute types.
"""
import ctypes as C

import numpy as np
import pytest

import nbk
import oracle
from helpers import ALL, PARAMS, mixed_box, real_slots, rms_rel

pytestmark = pytest.mark.gpu

NATOMS, SEED = 24000, 34
COT = 0.1                         # the energies' weight in L
GRAD_RMS_TOL = 1e-5               # gradients against the FP64 oracle (as the adjoint's own test)
# Central differences of the product's forward: a step moves one atom, so
# only the FP32 pair forces of its ~400 pairs change, each rounded to ~6e-8
# of itself; that rounding noise in L, ~1e-5 absolute, over a 2e-4 step is
# ~1e-1 against gradient components of 10-10^3, i.e. ~1e-3 relative.
FD_REL_TOL = 5e-3


class NonbondedFn:
    """torch.autograd.Function over one handle's refined tile lists."""

    def __new__(cls, *a, **k):
        raise TypeError("use NonbondedFn.apply")

    @staticmethod
    def make():
        import torch

        class _Fn(torch.autograd.Function):
            @staticmethod
            def forward(ctx, xyzq, run):
                # the handle keeps this device pointer for the adjoint: the
                # tensor stays alive in ctx until the backward has run
                ctx.xyzq = xyzq.detach()
                assert ctx.xyzq.is_contiguous()
                run.nb.force(run.packed, ALL, xyzq=ctx.xyzq, d_fixed=run.dX)
                ve = run.nb.virial_energy(ALL)
                X = run.dX.to(torch.float64) / nbk.FORCE_FIXED_SCALE
                F = X[:3].T.contiguous()
                S = X[3:].T.contiguous()
                E = torch.tensor([ve.energyVdw, ve.energyElec, ve.energySlow],
                                 dtype=torch.float64, device=xyzq.device)
                ctx.run = run
                return F, S, E

            @staticmethod
            def backward(ctx, gF, gS, gE):
                run = ctx.run
                n = run.packed.atomStorageSize
                wF = torch.zeros((n, 4), dtype=torch.float32, device=gF.device)
                wS = torch.zeros((n, 4), dtype=torch.float32, device=gF.device)
                wF[:, :3] = gF.to(torch.float32)
                wS[:, :3] = gS.to(torch.float32)
                cE = gE.detach().cpu().numpy()
                g = torch.zeros((n, 4), dtype=torch.float32, device=gF.device)
                run.gradAB.zero_()
                # the bound positions are the forward's: nothing ran in between
                run.nb.adjoint(wF, wS, float(cE[0]), float(cE[1]), float(cE[2]), g, run.gradAB,
                               type_mask=run.mask)
                return g, None

        return _Fn


class Run:
    def __init__(self, system, packed, lj=None):
        import torch
        self.packed = packed
        self.lj = system.lj_table() if lj is None else lj
        self.nb = nbk.Nonbonded(PARAMS, self.lj)
        self.nb.setup(packed)
        n = packed.atomStorageSize
        self.dX = torch.zeros((6, n), dtype=torch.int64, device="cuda")
        dim = self.lj[0]
        self.mask = np.zeros(dim, dtype=np.int32)
        self.mask[:dim - 2] = 1                 # the solute types; water O/H are fixed
        self.gradAB = torch.zeros(2 * dim * dim, dtype=torch.float64, device="cuda")
        self.x0 = torch.from_numpy(packed.xyzq.copy()).cuda()
        self.nb.build_tile_lists(packed, xyzq=self.x0)
        self.nb.force(packed, ALL | nbk.NBK_PAIRLIST, xyzq=self.x0)

    def loss(self, xyzq, w):
        """L of the product's forward at xyzq (FP64 sums)."""
        import torch
        self.nb.force(self.packed, ALL, xyzq=xyzq, d_fixed=self.dX)
        ve = self.nb.virial_energy(ALL)
        X = self.dX.to(torch.float64) / nbk.FORCE_FIXED_SCALE
        return float((w * X[:3].T).sum() + (w * X[3:].T).sum()) + COT * (
            ve.energyVdw + ve.energyElec + ve.energySlow)


def lj_with(system, sigma, epsilon):
    """The system's LJ table with per-type sigma / epsilon replaced."""
    nt = len(sigma)
    A, B, A14, B14 = (np.zeros(nt * nt) for _ in range(4))
    sg = np.ascontiguousarray(sigma, dtype=np.float64)
    ep = np.ascontiguousarray(epsilon, dtype=np.float64)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    rc = nbk.host_lib().nbk_lj_table(nt, dp(sg), dp(ep), 0, dp(A), dp(B), dp(A14), dp(B14))
    assert rc == 0
    return nt, A, B, A14, B14


@pytest.fixture(scope="module")
def case():
    import torch
    s = mixed_box(seed=SEED, natoms=NATOMS)
    p = nbk.Packed(s)
    n = p.atomStorageSize
    rng = np.random.default_rng(35)
    w = np.zeros((n, 3))
    w[real_slots(p)] = rng.standard_normal((int(real_slots(p).sum()), 3))
    run = Run(s, p)
    Fn = NonbondedFn.make()
    x = run.x0.clone().requires_grad_(True)
    F, S, E = Fn.apply(x, run)
    wt = torch.from_numpy(w).cuda()
    L = (wt * F).sum() + (wt * S).sum() + COT * E.sum()
    (g,) = torch.autograd.grad(L, x)
    gab = run.gradAB.cpu().numpy()
    return dict(system=s, packed=p, w=w, run=run, L=float(L.detach()), grad=g.cpu().numpy(),
                gab=gab)


def test_autograd_gradient_matches_the_fp64_oracle(case):
    p, w = case["packed"], case["w"]
    o = oracle.Oracle(p, PARAMS)
    Lo, gX, gQ, gA, gB = o.adjoint(w, w, COT, COT, COT)
    real = real_slots(p)
    g = case["grad"].astype(np.float64)
    ex = rms_rel(g[real, :3], gX[real])
    eq = rms_rel(g[real, 3], gQ[real])
    print(f"autograd vs FP64 oracle: positions {ex:.2e}, charges {eq:.2e}, "
          f"L {case['L']:.9e} vs {Lo:.9e}")
    assert ex <= GRAD_RMS_TOL and eq <= GRAD_RMS_TOL
    assert abs(case["L"] - Lo) <= 1e-6 * abs(Lo)


def _pick_slots(p, o, k, seed):
    """k real atom slots with no pair within 1e-3 A of the cutoff (a step could
    move such a pair across it)."""
    rng = np.random.default_rng(seed)
    out = []
    for slot in rng.permutation(p.slotOfAtom):
        if o.near_cutoff(int(slot), 1e-3) == 0:
            out.append(int(slot))
        if len(out) == k:
            break
    return out


def test_central_differences_of_the_product_forward(case):
    import torch
    p, w, run = case["packed"], case["w"], case["run"]
    o = oracle.Oracle(p, PARAMS)
    wt = torch.from_numpy(w).cuda()
    g = case["grad"].astype(np.float64)
    qscale = float(np.sqrt(332.0636 * PARAMS.scaling))
    fd, an = [], []
    for slot in _pick_slots(p, o, 6, 36):
        for comp, h in ((0, 1e-4), (1, 1e-4), (2, 1e-4), (3, 1e-4 * qscale)):
            xp = run.x0.clone()
            xm = run.x0.clone()
            xp[slot, comp] += h
            xm[slot, comp] -= h
            step = float(xp[slot, comp] - xm[slot, comp])   # the FP32 step actually taken
            fd.append((run.loss(xp, wt) - run.loss(xm, wt)) / step)
            an.append(g[slot, comp])
    fd, an = np.array(fd), np.array(an)
    err = np.abs(fd - an) / np.maximum(np.abs(an), 1e-3 * np.abs(an).max())
    print("central differences vs autograd (positions, scaled charges): max rel "
          f"{err.max():.2e}, norm rel {np.linalg.norm(fd - an) / np.linalg.norm(an):.2e}")
    assert np.linalg.norm(fd - an) <= FD_REL_TOL * np.linalg.norm(an)
    # restore the handle's lists and positions for the next test
    run.nb.force(p, ALL, xyzq=run.x0)


def test_lj_parameter_gradient_by_central_differences(case):
    import torch
    s, p, w = case["system"], case["packed"], case["w"]
    a = s.arrays()
    dim = len(a["sigma"])
    gab = case["gab"]
    gA, gB = gab[:dim * dim].reshape(dim, dim), gab[dim * dim:].reshape(dim, dim)
    gs, ge = nbk.lj_param_grad(a["sigma"], a["epsilon"], gA, gB, PARAMS.scaling)
    wt = torch.from_numpy(w).cuda()
    fd, an = [], []
    for t in (0, 5, 17):                  # solute types
        for which, grad in (("sigma", gs), ("epsilon", ge)):
            vals = []
            for sign in (1.0, -1.0):
                sig, eps = a["sigma"].copy(), a["epsilon"].copy()
                (sig if which == "sigma" else eps)[t] += sign * 1e-5
                r = Run(s, p, lj=lj_with(s, sig, eps))
                vals.append(r.loss(r.x0, wt))
                r.nb.close()
            fd.append((vals[0] - vals[1]) / 2e-5)
            an.append(grad[t])
    fd, an = np.array(fd), np.array(an)
    print(f"LJ parameter gradients: central differences {fd}, adjoint {an}")
    assert np.linalg.norm(fd - an) <= FD_REL_TOL * np.linalg.norm(an)
