"""Batched replicas (needs a B200): one handle evaluating several independent
systems gives, per replica, exactly what a separate handle gives."""
import numpy as np
import pytest

import nbk
import oracle
from helpers import ALL, FORCE_RMS_TOL, PARAMS, mixed_box, real_slots, rms_rel

pytestmark = pytest.mark.gpu

SIZES = (2000, 7000, 3100, 12000, 4500)


@pytest.fixture(scope="module")
def replicas():
    systems = [mixed_box(seed=40 + k, natoms=n) for k, n in enumerate(SIZES)]
    return systems, nbk.Packed.many(systems)


def _single(system, flags):
    import torch
    p = nbk.Packed(system)
    nb = nbk.Nonbonded(PARAMS, system.lj_table())
    nb.setup(p)
    X = torch.zeros((6, p.atomStorageSize), dtype=torch.int64, device="cuda")
    nb.build_tile_lists(p)
    nb.force(p, flags | nbk.NBK_PAIRLIST, xyzq=p.xyzq, d_fixed=X)
    nb.force(p, flags, xyzq=p.xyzq, d_fixed=X)
    ve = nb.virial_energy(flags)
    counts = nb.pair_count()
    return X.cpu().numpy(), ve, counts, p


@pytest.mark.parametrize("corr", [False, True])
def test_batch_equals_single_handles(replicas, corr):
    import torch
    systems, many = replicas
    flags = ALL | (nbk.NBK_CORRECTIONS if corr else 0)
    nb = nbk.Nonbonded(PARAMS, systems[0].lj_table())
    nb.setup(many)
    nb.set_replicas(many)
    X = torch.zeros((6, many.atomStorageSize), dtype=torch.int64, device="cuda")
    nb.build_tile_lists(many)
    nb.force(many, flags | nbk.NBK_PAIRLIST, xyzq=many.xyzq, d_fixed=X)
    nb.force(many, flags, xyzq=many.xyzq, d_fixed=X)
    ves = nb.virial_energy_batch()
    counts = nb.pair_counts()
    Xb = X.cpu().numpy()
    ss = many.replicaSlotStart
    for r, s in enumerate(systems):
        Xs, ve, cnt, p = _single(s, flags)
        assert np.array_equal(Xb[:, ss[r]:ss[r + 1]], Xs), r
        for k in ("energyVdw", "energyElec", "energySlow"):
            assert getattr(ves[r], k) == getattr(ve, k), (r, k)
        assert list(ves[r].virial) == list(ve.virial), r
        assert list(ves[r].virialSlow) == list(ve.virialSlow), r
        assert counts[r] == cnt, r


def test_batch_replica_against_oracle(replicas):
    import torch
    systems, many = replicas
    nb = nbk.Nonbonded(PARAMS, systems[0].lj_table())
    nb.setup(many)
    nb.set_replicas(many)
    X = torch.zeros((6, many.atomStorageSize), dtype=torch.int64, device="cuda")
    nb.build_tile_lists(many)
    nb.force(many, ALL | nbk.NBK_PAIRLIST, xyzq=many.xyzq, d_fixed=X)
    r = 3
    p = nbk.Packed(systems[r])
    Fo, So, ro = oracle.Oracle(p, PARAMS).forces(1)
    ss = many.replicaSlotStart
    F = X[:3, ss[r]:ss[r + 1]].T.cpu().numpy() / nbk.FORCE_FIXED_SCALE
    real = real_slots(p)
    assert rms_rel(F[real], Fo[real]) <= FORCE_RMS_TOL
    assert nb.pair_counts()[r] == ro["pairs"]


def test_batch_rejects_fp64_energy(replicas):
    systems, many = replicas
    nb = nbk.Nonbonded(PARAMS, systems[0].lj_table())
    nb.setup(many)
    nb.set_replicas(many)
    nb.build_tile_lists(many)
    with pytest.raises(nbk.NbkError, match="not available with replicas"):
        nb.force(many, ALL | nbk.NBK_PAIRLIST | nbk.NBK_ENERGY_FP64, xyzq=many.xyzq)
