"""Replica packing (nbk_pack_many): one concatenated layout for many systems."""
import numpy as np

import nbk
from helpers import mixed_box


def test_pack_many_offsets_match_single_packings():
    systems = [mixed_box(seed=20 + k, natoms=n) for k, n in enumerate((2400, 5100, 3300))]
    singles = [nbk.Packed(s) for s in systems]
    many = nbk.Packed.many(systems)
    assert many.numReplicas == 3
    ss = many.replicaSlotStart
    assert ss[0] == 0 and np.all(np.diff(ss) == [p.atomStorageSize for p in singles])
    assert many.atomStorageSize == ss[-1]
    pc = 0
    for r, p in enumerate(singles):
        sl = slice(ss[r], ss[r + 1])
        assert np.array_equal(many.xyzq[sl], p.xyzq)
        assert np.array_equal(many.vdwTypes[sl], p.vdwTypes)
        assert np.array_equal(many.atomIndex[sl], p.atomIndex + many.replicaAtomStart[r])
        np.testing.assert_array_equal(many.replicaLattice[r], p.lattice)
        nc = p.numComputes
        assert np.all(many.replicaOfCompute[pc:pc + nc] == r)
        assert np.array_equal(many.computes_patch[pc:pc + nc], p.computes_patch + sum(
            q.numPatches for q in singles[:r]))
        pc += nc
    # exclusion bases stay inside each replica's part of the concatenated bit array
    assert len(many.exclusionBits) == sum(len(p.exclusionBits) for p in singles)
    # tuple slots are offset into each replica's slot range
    nt = [len(p.excluded) for p in singles]
    t0 = 0
    for r, p in enumerate(singles):
        t = many.excluded[t0:t0 + nt[r]]
        assert np.array_equal(t["i"], p.excluded["i"] + ss[r])
        t0 += nt[r]
