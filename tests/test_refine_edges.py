"""Edge cases of the pairlist refinement: exclusion windows wider than the
kernel's FP32 index test covers (maxdiff above 2896), global atom indices at
or above 2^24, and fixed atoms (numFreeAtoms < numAtoms).

The renumbered and shifted systems carry the same exclusions under new global
indices, so the oracle's pair set must not change (checked on the CPU, which
validates the re-encoding); the GPU tests require the product's refined lists
-- and, where the reference kernels are built, the reference's -- to hold
exactly the oracle's pairs and excluded-pair count on each variant.
"""
import numpy as np
import pytest

import nbk
import oracle
import refgpu
from helpers import (ALL, PARAMS, GpuRun, mixed_box, molecule_boundaries, renumbered,
                     PackedVariant, reference_pairs, unordered_keys)

FP_WINDOW_MAX_DIFF = 2896   # largest maxdiff the kernel's FP32 window test covers


@pytest.fixture(scope="module")
def base():
    s = mixed_box(natoms=20000)
    p = nbk.Packed(s)
    return s, p, oracle.Oracle(p, PARAMS)


def interleaved(system, packed):
    """Solute chains renumbered 4-way interleaved: bonded neighbours end up
    ~1300-3900 indices apart, the waters keep their indices."""
    b = molecule_boundaries(system)
    m = int(b[(b >= system.natoms // 5) & (b % 4 == 0)][0])
    perm = np.arange(system.natoms)
    g = np.arange(m)
    perm[:m] = (g % 4) * (m // 4) + g // 4
    return renumbered(packed, perm)


def shifted(system, packed):
    """Global indices of the second half of the molecules moved above 2^24."""
    b = molecule_boundaries(system)
    cut = int(b[b >= system.natoms // 2][0])
    perm = np.arange(system.natoms) + np.where(np.arange(system.natoms) >= cut, (1 << 24) + 7, 0)
    return renumbered(packed, perm)


def with_fixed(packed):
    """Every third patch keeps its last quarter of atoms fixed."""
    pa = packed.patches.copy()
    for k in range(0, len(pa), 3):
        pa[k, 1] = pa[k, 0] - pa[k, 0] // 4
    return PackedVariant(packed, patches=pa)


def test_variants_keep_pairs(base):
    s, p, o = base
    keys, nex = o.pairs()
    v = interleaved(s, p)
    assert v.exclIndexMaxDiff[:, 1].max() > FP_WINDOW_MAX_DIFF
    assert (v.exclIndexMaxDiff[:, 1] <= FP_WINDOW_MAX_DIFF).any()
    w = shifted(s, p)
    assert w.atomIndex.max() >= (1 << 24) and w.atomIndex.min() < (1 << 24)
    for var in (v, w):
        k2, n2 = oracle.Oracle(var, PARAMS).pairs()
        assert n2 == nex
        assert np.array_equal(k2, keys)


def test_fixed_atoms_change_pairs(base):
    s, p, o = base
    keys, _ = o.pairs()
    k2, _ = oracle.Oracle(with_fixed(p), PARAMS).pairs()
    assert 0 < len(k2) < len(keys)
    assert np.isin(k2, keys).all()


def _check(var):
    keys, nex = oracle.Oracle(var, PARAMS).pairs()
    run = GpuRun(var)
    run.build()
    run.eval(ALL | nbk.NBK_PAIRLIST)
    tl, ja, ex = run.nb.export_tile_lists()
    mine = nbk.pairs_from_tile_lists(tl, ja, ex, var.atomStorageSize)
    assert len(np.unique(mine)) == len(mine), "pair listed twice"
    assert np.array_equal(mine, keys)
    assert run.nb.stat().numExcluded == nex
    if refgpu.available():
        ref = refgpu.RefGpu(PARAMS, var.system.lj_table(), do_table=1)
        ref.setup(var)
        rk, rnex, reruns = reference_pairs(ref, np.ascontiguousarray(var.xyzq),
                                           var.atomStorageSize)
        if reruns:
            print(f"reference lists re-evaluated {reruns}x (a pair listed twice)")
        assert np.array_equal(rk, unordered_keys(keys, var.atomStorageSize))
        assert rnex == nex
    print(f"pairs {len(keys)} excluded {nex}")


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["interleaved", "shifted", "fixed"])
def test_refine_edge_pairsets(base, which):
    s, p, _ = base
    var = {"interleaved": lambda: interleaved(s, p), "shifted": lambda: shifted(s, p),
           "fixed": lambda: with_fixed(p)}[which]()
    _check(var)
