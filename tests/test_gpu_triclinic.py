"""Parity on a triclinic cell (needs a B200). The kernels take general lattice
vectors, as the reference's do (the shift of a compute is offsetXYZ.x lata +
offsetXYZ.y latb + offsetXYZ.z latc, src/CudaComputeNonbondedKernel.cu:737-743,
formed here and in the oracle as the same FP32 FMA chain). The 20,000-atom
mixed system is sheared as a whole: every position and lattice vector is
mapped by r -> S r with S upper unitriangular, so that a stays along x and b in
the xy plane. Patch-centred coordinates, compute offsets in lattice units and
exclusions carry over unchanged. The shear is small enough that every patch's
perpendicular width stays above the pairlist distance (checked below), so every
pair within it still lies in a self or neighbour compute; the oracle and the
GPU then see the same non-orthogonal cell, and the pair set, forces, energies
and virials must agree as on the orthorhombic systems."""
import numpy as np
import pytest

import nbk
import oracle
import refgpu
from helpers import (ALL, ENERGY_TOL, FORCE_RMS_TOL, PARAMS, VIRIAL_TOL, GpuRun,
                     PackedVariant, compare, mixed_box, real_slots, reference_pairs, rel,
                     rms_rel, unordered_keys)

pytestmark = pytest.mark.gpu

# r -> S r: b gains 0.15 of its length along x, c 0.10 along x and 0.12 along y
SHEAR = np.array([[1.0, 0.15, 0.10],
                  [0.0, 1.0, 0.12],
                  [0.0, 0.0, 1.0]])


def sheared(packed, S):
    """The packed system with positions and lattice vectors mapped by S."""
    xyzq = np.array(packed.xyzq, dtype=np.float32, copy=True)
    xyzq[:, :3] = (xyzq[:, :3].astype(np.float64) @ S.T).astype(np.float32)
    v = PackedVariant(packed, xyzq=xyzq)
    L = (packed.lattice.astype(np.float64) @ S.T).astype(np.float32)  # rows a, b, c
    v.lattice = L
    for name, row in zip(("lata", "latb", "latc"), L):
        setattr(v.v, name, nbk.Float3(float(row[0]), float(row[1]), float(row[2])))
    return v


@pytest.fixture(scope="module")
def triclinic():
    s = mixed_box(natoms=20000)
    p = nbk.Packed(s)
    box = np.diag(p.lattice.astype(np.float64))
    per_dim = np.floor(box / PARAMS.pairlistdist)      # the packer's patch grid
    assert int(np.prod(per_dim)) == p.numPatches
    t = sheared(p, SHEAR)
    L = t.lattice.astype(np.float64)
    assert L[0, 1] == 0 and L[0, 2] == 0 and L[1, 2] == 0 and L[1, 0] > 0 and L[2, 0] > 0
    # perpendicular width of a patch along each lattice direction
    widths = 1.0 / np.linalg.norm(np.linalg.inv(L).T, axis=1) / per_dim
    assert widths.min() > PARAMS.pairlistdist, widths
    return s, t, oracle.Oracle(t, PARAMS)


def test_triclinic_pairset(triclinic):
    s, p, o = triclinic
    run = GpuRun(p)
    run.build()
    run.eval(ALL | nbk.NBK_PAIRLIST)
    tl, ja, ex = run.nb.export_tile_lists()
    keys = nbk.pairs_from_tile_lists(tl, ja, ex, p.atomStorageSize)
    ref, nex = o.pairs()
    assert len(np.unique(keys)) == len(keys), "pair listed twice"
    assert np.array_equal(keys, ref)
    assert run.nb.stat().numExcluded == nex


@pytest.mark.parametrize("corr", [False, True])
def test_triclinic_forces_energies_virials(triclinic, corr):
    s, p, o = triclinic
    extra = nbk.NBK_CORRECTIONS if corr else 0
    Fo, So, ro = o.forces(3 if corr else 1)
    run = GpuRun(p)
    run.build()
    real = real_slots(p)
    # the virials have off-diagonal parts now: compare them as whole tensors
    assert np.abs(ro["virial"] - ro["virial"].T).max() <= 1e-9 * np.abs(ro["virial"]).max()
    for flags in (ALL | nbk.NBK_PAIRLIST | extra, ALL | extra):
        F, S, res, _ = run.eval(flags)
        err = compare(F, S, res, Fo, So, ro, real)
        print(f"triclinic flags={flags} " + " ".join(f"{k}={v:.2e}" for k, v in err.items()))
        assert err["force"] <= FORCE_RMS_TOL and err["slow"] <= FORCE_RMS_TOL, err
        assert err["energyVdw"] <= ENERGY_TOL, err
        assert err["energyElec"] <= ENERGY_TOL and err["energySlow"] <= ENERGY_TOL, err
        assert err["virial"] <= VIRIAL_TOL and err["virialSlow"] <= VIRIAL_TOL, err


@pytest.mark.skipif(not refgpu.available(), reason="reference kernels not built (oracle/ref_gpu)")
def test_triclinic_reference_kernels(triclinic):
    """The reference's own CudaTileListKernel and CudaComputeNonbondedKernel on
    the same sheared cell: their refined pair set equals the oracle's, and their
    direct-math fast forces, LJ energy and virial (the reference allows direct
    math only without slow forces) agree with the oracle as they do on the
    orthorhombic systems. This pins the oracle's triclinic shifts and virial to
    the reference, not only to the product."""
    s, p, o = triclinic
    xyzq = np.ascontiguousarray(p.xyzq)
    tab = refgpu.RefGpu(PARAMS, s.lj_table(), do_table=1)  # its mode with slow forces
    tab.setup(p)
    ku, nexcl = reference_pairs(tab, xyzq, p.atomStorageSize)
    ok, nex = o.pairs()
    assert np.array_equal(ku, unordered_keys(ok, p.atomStorageSize))
    assert nexcl == nex
    del tab
    ref = refgpu.RefGpu(PARAMS, s.lj_table(), do_table=0)
    ref.setup(p)
    Fo, So, ro = o.forces(1)
    real = real_slots(p)
    for pl in (1, 0):
        ref.eval(pl, 1, 1, 0, xyzq)
        F, S, ve = ref.results()
        e = dict(force=rms_rel(F[real, :3].astype(np.float64), Fo[real]),
                 energyVdw=rel(ve[18], ro["energyVdw"]),
                 virial=rms_rel(ve[:9].reshape(3, 3), ro["virial"]))
        print(f"reference direct math, triclinic, pairlist={pl}: "
              + " ".join(f"{k}={v:.2e}" for k, v in e.items()))
        assert e["force"] <= FORCE_RMS_TOL and e["virial"] <= 1e-5 and e["energyVdw"] <= 1e-5, e
