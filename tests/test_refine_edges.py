"""Edge cases of the pairlist refinement: exclusion windows wider than the
kernel's FP32 index test covers (maxdiff above 2896), global atom indices at
or above 2^24, fixed atoms (numFreeAtoms < numAtoms), and pairs placed exactly
on the pair rule's edges (r^2 equal to plcutoff^2 or cutoff^2 in FP32, and one
FP32 step inside).

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


PLCUTOFF, CUTOFF = 13.5, 12.0
# (x_i, x_j) of the four placed pairs, both atoms in patch 0 with equal y and
# z: |dx| = 13.5 (r^2 = plcutoff^2: not listed), 13.5 - 2^-20 (listed), 12
# (r^2 = cutoff^2: listed, not interacting), 12 - 2^-20 (interacting). Every
# value and difference is exact in FP32.
EDGE_X = [(-6.75, 6.75), (-6.75 + 2.0 ** -20, 6.75), (-6.0, 6.0), (-6.0 + 2.0 ** -20, 6.0)]


def on_edges(system, packed):
    """Eight water oxygens of patch 0 moved to form the EDGE_X pairs; returns
    the variant and the slot pairs."""
    x = packed.xyzq.copy()
    n, start = int(packed.patches[0, 0]), int(packed.patches[0, 2])
    slots = np.arange(start, start + n)
    oxygen = system.lj_table()[0] - 2          # water O type of the mixed systems
    ox = [int(a) for a in slots if packed.vdwTypes[a] == oxygen][:8]
    assert len(ox) == 8
    moved = set(ox)
    rest = np.array([a for a in slots if a not in moved])
    grid = [(y, z) for y in np.arange(-6.0, 6.5, 1.5) for z in np.arange(-6.0, 6.5, 1.5)]
    pairs, used = [], []
    for m, (xi, xj) in enumerate(EDGE_X):
        for y, z in grid:
            if any(abs(y - u) < 2.0 and abs(z - v) < 2.0 for u, v in used):
                continue
            cand = np.array([[xi, y, z], [xj, y, z]], np.float32)
            d = np.linalg.norm(x[rest, None, :3] - cand[None], axis=2).min()
            if d > 1.2:
                break
        else:
            raise AssertionError("no free place for an edge pair")
        used.append((y, z))
        a, b = ox[2 * m], ox[2 * m + 1]
        x[a, :3], x[b, :3] = cand[0], cand[1]
        pairs.append((a, b))
    return PackedVariant(packed, xyzq=x), pairs


def _edge_keys(var, pairs):
    n = np.uint64(var.atomStorageSize)
    return [np.uint64(min(a, b)) * n + np.uint64(max(a, b)) for a, b in pairs]


def test_edge_pairs_fall_on_designed_sides(base):
    s, p, _ = base
    var, pairs = on_edges(s, p)
    r2 = [np.float32(var.xyzq[b, 0] - var.xyzq[a, 0]) ** 2 for a, b in pairs]
    assert r2[0] == np.float32(PLCUTOFF) ** 2 and r2[1] < np.float32(PLCUTOFF) ** 2
    assert r2[2] == np.float32(CUTOFF) ** 2 and r2[3] < np.float32(CUTOFF) ** 2
    keys, _ = oracle.Oracle(var, PARAMS).pairs()
    listed = np.isin(_edge_keys(var, pairs), unordered_keys(keys, var.atomStorageSize))
    assert listed.tolist() == [False, True, True, True]


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
        rk, rnex = reference_pairs(ref, np.ascontiguousarray(var.xyzq), var.atomStorageSize)
        assert np.array_equal(rk, unordered_keys(keys, var.atomStorageSize))
        assert rnex == nex
    print(f"pairs {len(keys)} excluded {nex}")
    return run


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["interleaved", "shifted", "fixed", "edges"])
def test_refine_edge_pairsets(base, which):
    s, p, _ = base
    var = {"interleaved": lambda: interleaved(s, p), "shifted": lambda: shifted(s, p),
           "fixed": lambda: with_fixed(p), "edges": lambda: on_edges(s, p)[0]}[which]()
    run = _check(var)
    if which == "edges":
        # interacting pairs (r^2 < cutoff^2 in FP32) counted by the force
        # kernel equal the oracle's count on the same positions
        run.eval(ALL)
        _, _, ro = oracle.Oracle(var, PARAMS).forces(1)
        assert run.nb.pair_count() == int(ro["pairs"])
