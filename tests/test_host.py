"""Host-side input preparation (the mirror of CudaComputeNonbonded's packing)."""
import numpy as np
import pytest

import nbk
from helpers import mixed_box, water_box


@pytest.fixture(scope="module")
def mixed():
    s = mixed_box(seed=5, natoms=12000)
    return s, nbk.Packed(s)


def test_generator_is_seeded_and_neutral():
    a = mixed_box(seed=3, natoms=6000).arrays()
    b = mixed_box(seed=3, natoms=6000).arrays()
    c = mixed_box(seed=4, natoms=6000).arrays()
    assert np.array_equal(a["pos"], b["pos"]) and not np.array_equal(a["pos"], c["pos"])
    assert abs(a["charge"].sum()) < 1e-9
    assert a["numSolute"] + 3 * a["numWaters"] == 6000
    assert abs(a["numSolute"] / 6000 - 0.3) < 0.01
    box = a["box"]
    assert np.all(a["pos"] >= 0) and np.all(a["pos"] < box)
    # density 0.1 atoms / A^3 when the box is sized automatically
    assert abs(6000 / np.prod(box) - 0.1) < 1e-9


def test_water_geometry():
    a = water_box(seed=1, nwater=200, box=20.0).arrays()
    pos, box = a["pos"], a["box"]
    o, h1, h2 = pos[0::3], pos[1::3], pos[2::3]

    def mi(d):
        return d - box * np.round(d / box)
    r1 = np.linalg.norm(mi(h1 - o), axis=1)
    r2 = np.linalg.norm(mi(h2 - o), axis=1)
    np.testing.assert_allclose(r1, 0.9572, atol=1e-9)
    np.testing.assert_allclose(r2, 0.9572, atol=1e-9)
    cosang = (mi(h1 - o) * mi(h2 - o)).sum(1) / (r1 * r2)
    np.testing.assert_allclose(np.degrees(np.arccos(cosang)), 104.52, atol=1e-6)


def test_patch_layout(mixed):
    s, p = mixed
    pt = p.patches
    assert np.all(pt[:, 2] % 32 == 0)
    padded = ((pt[:, 0] + 31) // 32) * 32
    assert np.array_equal(pt[1:, 2], (pt[:-1, 2] + padded[:-1]))
    assert pt[:, 0].sum() == s.natoms
    assert p.atomStorageSize == pt[-1, 2] + padded[-1]
    # every atom sits in exactly one slot; padding repeats the patch's last atom
    assert len(np.unique(p.slotOfAtom)) == s.natoms
    for k in range(len(pt)):
        n, start = pt[k, 0], pt[k, 2]
        for slot in range(start + n, start + padded[k]):
            assert np.array_equal(p.xyzq[slot], p.xyzq[start + n - 1])
            assert p.atomIndex[slot] == p.atomIndex[start + n - 1]


def test_patch_centred_coordinates(mixed):
    s, p = mixed
    a = s.arrays()
    cell = a["box"] / np.array(p.v.patchGrid)
    assert np.all(np.abs(p.xyzq[:, :3]) <= 0.5 * cell + 1e-4)
    # q = charge * sqrt(332.0636)
    slot = p.slotOfAtom
    np.testing.assert_allclose(p.xyzq[slot, 3], a["charge"] * np.sqrt(332.0636), rtol=1e-6,
                               atol=1e-6)


def test_tiles_are_compact(mixed):
    """Recursive bisection gives 32-atom tiles much smaller than a patch."""
    s, p = mixed
    ext = []
    for k in range(len(p.patches)):
        n, start = p.patches[k, 0], p.patches[k, 2]
        for t in range(0, n - 31, 32):
            x = p.xyzq[start + t:start + t + 32, :3]
            ext.append((x.max(0) - x.min(0)).mean())
    cell = (s.arrays()["box"] / np.array(p.v.patchGrid)).mean()
    assert np.mean(ext) < 0.6 * cell


def test_computes_are_self_plus_half_shell(mixed):
    s, p = mixed
    g = np.array(p.v.patchGrid)
    assert p.numComputes == 14 * p.numPatches
    keys = {(int(a), int(b), *np.round(o * g).astype(int)) for (a, b), o in
            zip(p.computes_patch, p.computes_offset)}
    assert len(keys) == p.numComputes
    # offsets are -d/n for neighbour displacements d in {-1,0,1}^3, upper half
    d = -np.round(p.computes_offset * g).astype(int)
    assert np.all(np.abs(d) <= 1)
    lex = d[:, 2] * 9 + d[:, 1] * 3 + d[:, 0]
    assert np.all(lex >= 0)


def test_exclusion_bits_encode_full_exclusions(mixed):
    """Decoding the bit array with the kernel's rule gives exactly the 1-2/1-3
    pairs (and self) of every atom (CudaComputeNonbonded::buildExclusions)."""
    s, p = mixed
    a = s.arrays()
    partners = {}
    for x, y in a["fullExcl"]:
        partners.setdefault(x, set()).add(y)
        partners.setdefault(y, set()).add(x)
    bits = p.exclusionBits
    slot = p.slotOfAtom

    def excluded(i, j):
        base, maxdiff = p.exclIndexMaxDiff[slot[i]]
        d = j - i
        if abs(d) > maxdiff:
            return False
        b = d + base
        return bool((bits[b >> 5] >> (b & 31)) & 1)

    for i in range(0, s.natoms, 7):
        want = partners.get(i, set()) | {i}
        lo, hi = max(0, i - 4), min(s.natoms, i + 5)
        for j in range(lo, hi):
            assert excluded(i, j) == (j in want), (i, j)
    # 1-4 pairs are not excluded (the nonbonded kernel computes them at full strength)
    for x, y in a["modPairs"][:200]:
        assert not excluded(x, y)


def test_correction_tuples_use_minimum_image(mixed):
    s, p = mixed
    for tup in (p.excluded, p.modified):
        xi = p.xyzq[tup["i"], :3].astype(np.float64)
        xj = p.xyzq[tup["j"], :3].astype(np.float64)
        sh = tup["off"].astype(np.float64) * np.diag(p.lattice).astype(np.float64)
        r = np.linalg.norm(xi + sh - xj, axis=1)
        assert r.max() < 5.0


def test_lj_table_combining():
    s = mixed_box(seed=3, natoms=6000)
    dim, A, B, A14, B14 = s.lj_table()
    a = s.arrays()
    sig, eps = a["sigma"], a["epsilon"]
    i, j = 3, 17
    sij = 0.5 * (sig[i] + sig[j])
    eij = np.sqrt(eps[i] * eps[j])
    assert np.isclose(B[i * dim + j], 4 * eij * sij ** 6, rtol=1e-14)
    assert np.isclose(A[i * dim + j], 4 * eij * sij ** 12, rtol=1e-14)
    assert np.array_equal(A.reshape(dim, dim), A.reshape(dim, dim).T)
    # hydrogen (last type) has no LJ
    assert np.all(A.reshape(dim, dim)[-1] == 0)
