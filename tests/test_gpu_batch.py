"""Batched replicas (needs a B200): one handle evaluating several independent
systems gives, per replica, exactly what a separate handle gives."""
import numpy as np
import pytest

import nbk
import oracle
from helpers import (ALL, ENERGY_TOL, FORCE_RMS_TOL, PARAMS, VIRIAL_TOL, compare, mixed_box,
                     real_slots)

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


@pytest.mark.parametrize("corr", [False, True])
def test_batch_replicas_against_oracle(replicas, corr):
    """Every replica of one batched evaluation against its own FP64 oracle:
    forces, and energies and virials at 1e-6, on the pairlist step and on a
    steady step."""
    import torch
    systems, many = replicas
    flags = ALL | (nbk.NBK_CORRECTIONS if corr else 0)
    nb = nbk.Nonbonded(PARAMS, systems[0].lj_table())
    nb.setup(many)
    nb.set_replicas(many)
    X = torch.zeros((6, many.atomStorageSize), dtype=torch.int64, device="cuda")
    nb.build_tile_lists(many)
    ss = many.replicaSlotStart
    for step in (flags | nbk.NBK_PAIRLIST, flags):
        nb.force(many, step, xyzq=many.xyzq, d_fixed=X)
        ves = nb.virial_energy_batch()
        counts = nb.pair_counts()
        Xb = X.cpu().numpy()
        for r, system in enumerate(systems):
            p = nbk.Packed(system)
            Fo, So, ro = oracle.Oracle(p, PARAMS).forces(3 if corr else 1)
            real = real_slots(p)
            F = Xb[:3, ss[r]:ss[r + 1]].T / nbk.FORCE_FIXED_SCALE
            S = Xb[3:, ss[r]:ss[r + 1]].T / nbk.FORCE_FIXED_SCALE
            res = dict(energyVdw=ves[r].energyVdw, energyElec=ves[r].energyElec,
                       energySlow=ves[r].energySlow,
                       virial=np.array(ves[r].virial).reshape(3, 3),
                       virialSlow=np.array(ves[r].virialSlow).reshape(3, 3))
            err = compare(F, S, res, Fo, So, ro, real)
            assert err["force"] <= FORCE_RMS_TOL and err["slow"] <= FORCE_RMS_TOL, (r, err)
            for k in ("energyVdw", "energyElec", "energySlow"):
                assert err[k] <= ENERGY_TOL, (r, k, err)
            assert err["virial"] <= VIRIAL_TOL and err["virialSlow"] <= VIRIAL_TOL, (r, err)
            assert counts[r] == ro["pairs"], r
