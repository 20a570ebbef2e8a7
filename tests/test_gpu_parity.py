"""Parity of the GPU path with the FP64 oracle (needs a B200)."""
import numpy as np
import pytest

import nbk
import oracle
from helpers import (ALL, ENERGY_TOL, FORCE_RMS_TOL, PARAMS, VIRIAL_TOL, GpuRun, compare,
                     mixed_box, real_slots, water_box)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def water():
    s = water_box()
    p = nbk.Packed(s)
    return s, p, oracle.Oracle(p, PARAMS)


@pytest.fixture(scope="module")
def mixed():
    s = mixed_box(natoms=20000)
    p = nbk.Packed(s)
    return s, p, oracle.Oracle(p, PARAMS)


def _pairset_check(p, o):
    run = GpuRun(p)
    run.build()
    run.eval(ALL | nbk.NBK_PAIRLIST)
    tl, ja, ex = run.nb.export_tile_lists()
    keys = nbk.pairs_from_tile_lists(tl, ja, ex, p.atomStorageSize)
    ref, nex = o.pairs()
    assert len(np.unique(keys)) == len(keys), "pair listed twice"
    assert len(keys) == len(ref)
    assert np.array_equal(keys, ref)
    st = run.nb.stat()
    assert st.numExcluded == nex


def test_pairset_water(water):
    _pairset_check(water[1], water[2])


def test_pairset_mixed(mixed):
    _pairset_check(mixed[1], mixed[2])


@pytest.mark.parametrize("corr", [False, True])
def test_forces_water(water, corr):
    s, p, o = water
    mode = 3 if corr else 1
    extra = nbk.NBK_CORRECTIONS if corr else 0
    Fo, So, ro = o.forces(mode)
    run = GpuRun(p)
    run.build()
    real = real_slots(p)
    for flags in (ALL | nbk.NBK_PAIRLIST | extra, ALL | extra):
        F, S, res, _ = run.eval(flags)
        err = compare(F, S, res, Fo, So, ro, real)
        print(flags, err)
        assert err["force"] <= FORCE_RMS_TOL and err["slow"] <= FORCE_RMS_TOL
        for k in ("energyVdw", "energyElec", "energySlow"):
            assert err[k] <= ENERGY_TOL, (k, err)
        assert err["virial"] <= VIRIAL_TOL and err["virialSlow"] <= VIRIAL_TOL, err


@pytest.mark.parametrize("corr", [False, True])
def test_forces_mixed(mixed, corr):
    s, p, o = mixed
    mode = 3 if corr else 1
    extra = nbk.NBK_CORRECTIONS if corr else 0
    Fo, So, ro = o.forces(mode)
    run = GpuRun(p)
    run.build()
    real = real_slots(p)
    for flags in (ALL | nbk.NBK_PAIRLIST | extra, ALL | extra):
        F, S, res, _ = run.eval(flags)
        err = compare(F, S, res, Fo, So, ro, real)
        print(flags, err)
        assert err["force"] <= FORCE_RMS_TOL and err["slow"] <= FORCE_RMS_TOL
        for k in ("energyVdw", "energyElec", "energySlow"):
            assert err[k] <= ENERGY_TOL, (k, err)
        assert err["virial"] <= VIRIAL_TOL and err["virialSlow"] <= VIRIAL_TOL, err


def test_deterministic(mixed):
    s, p, o = mixed
    run = GpuRun(p)
    run.build()
    _, _, r1, X1 = run.eval(ALL | nbk.NBK_PAIRLIST | nbk.NBK_CORRECTIONS)
    _, _, r2, X2 = run.eval(ALL | nbk.NBK_CORRECTIONS)
    _, _, r3, X3 = run.eval(ALL | nbk.NBK_CORRECTIONS)
    assert np.array_equal(X1, X2) and np.array_equal(X2, X3)
    for k in ("energyVdw", "energyElec", "energySlow"):
        assert r1[k] == r2[k] == r3[k]
    assert np.array_equal(r1["virial"], r3["virial"])
