"""GPU adjoint (needs a B200) against the FP64 oracle's analytic gradient
(itself pinned to central differences in tests/test_oracle_adjoint.py)."""
import numpy as np
import pytest

import nbk
import oracle
from helpers import ALL, PARAMS, mixed_box, real_slots, rms_rel

pytestmark = pytest.mark.gpu

GRAD_RMS_TOL = 1e-5


@pytest.fixture(scope="module")
def case():
    import torch
    s = mixed_box(seed=33, natoms=12000)
    p = nbk.Packed(s)
    n = p.atomStorageSize
    rng = np.random.default_rng(3)
    w = rng.standard_normal((n, 3)).astype(np.float32)
    w4 = np.zeros((n, 4), dtype=np.float32)
    w4[:, :3] = w
    o = oracle.Oracle(p, PARAMS)
    L, gX, gQ, gA, gB = o.adjoint(w.astype(np.float64), w.astype(np.float64), 0.1, 0.1, 0.1)
    nb = nbk.Nonbonded(PARAMS, s.lj_table())
    nb.setup(p)
    nb.build_tile_lists(p)
    nb.force(p, ALL | nbk.NBK_PAIRLIST, xyzq=p.xyzq)
    dim = s.lj_table()[0]
    mask = np.zeros(dim, dtype=np.int32)
    mask[:dim - 2] = 1                    # the 32 solute types; water O/H are fixed
    dw = torch.from_numpy(w4).cuda()
    g = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    gab = torch.zeros(2 * dim * dim, dtype=torch.float64, device="cuda")
    nb.adjoint(dw, dw, 0.1, 0.1, 0.1, g, gab, type_mask=mask)
    torch.cuda.synchronize()
    return s, p, dict(gX=gX, gQ=gQ, gA=gA, gB=gB), g.cpu().numpy(), gab.cpu().numpy(), mask


def test_position_and_charge_gradients(case):
    s, p, ref, g, gab, mask = case
    real = real_slots(p)
    ex = rms_rel(g[real, :3].astype(np.float64), ref["gX"][real])
    eq = rms_rel(g[real, 3].astype(np.float64), ref["gQ"][real])
    print(f"adjoint: position grad rms rel {ex:.2e}, charge grad rms rel {eq:.2e}")
    assert ex <= GRAD_RMS_TOL and eq <= GRAD_RMS_TOL


def test_lj_parameter_gradients(case):
    s, p, ref, g, gab, mask = case
    dim = len(mask)
    gA = gab[:dim * dim].reshape(dim, dim)
    gB = gab[dim * dim:].reshape(dim, dim)
    keep = (mask[:, None] | mask[None, :]).astype(bool)
    rA, rB = np.where(keep, ref["gA"], 0.0), np.where(keep, ref["gB"], 0.0)
    assert rms_rel(gA, rA) <= 1e-4 and rms_rel(gB, rB) <= 1e-4
    a = s.arrays()
    gs, ge = nbk.lj_param_grad(a["sigma"], a["epsilon"], gA, gB, PARAMS.scaling)
    rs, re_ = nbk.lj_param_grad(a["sigma"], a["epsilon"], rA, rB, PARAMS.scaling)
    sol = slice(0, dim - 2)
    print(f"sigma grad rms rel {rms_rel(gs[sol], rs[sol]):.2e}, eps {rms_rel(ge[sol], re_[sol]):.2e}")
    assert rms_rel(gs[sol], rs[sol]) <= 1e-4 and rms_rel(ge[sol], re_[sol]) <= 1e-4
