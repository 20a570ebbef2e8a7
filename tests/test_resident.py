"""GPU-resident input marshaling (nbk_sort_patch_atoms, nbk_set_compute_positions,
nbk_update_vdw_types_excl_device).

CPU: the buffer-order layout helper and a numpy restatement of the three
kernels reproduce the host packing (nbk_pack) -- positions bit for bit, the
bisection order block for block.
GPU: the kernels against those restatements, bit for bit; the whole
device-resident pipeline (device sort -> positions -> types -> tile lists ->
forces) against the oracle, as atom pairs and per-atom forces.
"""
import numpy as np
import pytest

import nbk
import oracle
from helpers import ALL, ENERGY_TOL, FORCE_RMS_TOL, PARAMS, mixed_box, rms_rel


@pytest.fixture(scope="module")
def system():
    s = mixed_box(natoms=20000)
    p = nbk.Packed(s)
    return s, p


def restate_positions(L, order, storage):
    """numpy form of nbk_set_compute_positions for an identity lattice."""
    xyzq = np.zeros((storage, 4), np.float32)
    for q in range(L.numPatches):
        b, nb, n, npad = L.records[q, 1], L.records[q, 2], L.records[q, 3], L.records[q, 4]
        if n == 0:
            continue
        a = b + order[b + np.minimum(np.arange(npad), n - 1)]
        xyzq[nb:nb + npad, :3] = (L.pos[:, a].T - L.centres[q]).astype(np.float32)
        xyzq[nb:nb + npad, 3] = (L.charge[a].astype(np.float64) * L.qscale).astype(np.float32)
    return xyzq


def restate_slots(L, order, storage):
    """Global atom id of every slot (padding repeats the patch's last atom)."""
    ids = np.full(storage, -1, np.int64)
    for q in range(L.numPatches):
        b, nb, n, npad = L.records[q, 1], L.records[q, 2], L.records[q, 3], L.records[q, 4]
        if n == 0:
            continue
        ids[nb:nb + npad] = L.ids[b + order[b + np.minimum(np.arange(npad), n - 1)]]
    return ids


def block_sets(slot_ids, packed, width=8):
    """Sorted atom ids of every `width`-slot block of real atoms, per patch."""
    out = []
    for n, _, start, _ in packed.patches:
        for k in range(0, n, width):
            out.append(tuple(sorted(slot_ids[start + k:start + min(k + width, n)])))
    return out


def test_layout_restates_host_packing(system):
    s, p = system
    L = nbk.ResidentLayout(s, p, device=None, shuffle_seed=3)
    order = L.host_sort_order(p)
    xyzq = restate_positions(L, order, p.atomStorageSize)
    assert np.array_equal(xyzq[:, :3], p.xyzq[:, :3])
    # charges enter as FP32 (as the integrator's do), so q is compared to that form
    slot_ids = restate_slots(L, order, p.atomStorageSize)
    assert np.array_equal(slot_ids, p.atomIndex)
    a = s.arrays()
    want_q = (np.asarray(a["charge"], np.float32)[slot_ids].astype(np.float64) *
              L.qscale).astype(np.float32)
    assert np.array_equal(xyzq[:, 3], want_q)
    assert np.array_equal(L.excl_by_atom[slot_ids][:, ::-1], p.exclIndexMaxDiff)
    assert np.array_equal(np.asarray(a["type"], np.int32)[slot_ids], p.vdwTypes)


@pytest.mark.gpu
def test_device_sort_matches_bisection(system):
    import torch
    s, p = system
    L = nbk.ResidentLayout(s, p, shuffle_seed=5)
    order = torch.zeros(len(L.ids), dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    L.sort_patch_atoms(order, status=status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    o = order.cpu().numpy()
    for q in range(L.numPatches):  # a permutation of every patch
        b, n = L.records[q, 1], L.records[q, 3]
        assert np.array_equal(np.sort(o[b:b + n]), np.arange(n))
    dev_ids = restate_slots(L, o, p.atomStorageSize)
    assert block_sets(dev_ids, p) == block_sets(p.atomIndex, p)
    # a bound below the largest patch leaves those patches in buffer order and counts them
    m = int(L.records[:, 3].max())
    status.zero_()
    L.sort_patch_atoms(order, max_patch_atoms=m - 1, status=status)
    torch.cuda.synchronize()
    big = int((L.records[:, 3] > m - 1).sum())
    assert int(status.item()) == big


@pytest.mark.gpu
def test_device_positions_and_types_bit_exact(system):
    import torch
    s, p = system
    L = nbk.ResidentLayout(s, p, shuffle_seed=7)
    order_h = L.host_sort_order(p)
    order = torch.from_numpy(order_h).cuda()
    xyzq = torch.zeros((p.atomStorageSize, 4), dtype=torch.float32, device="cuda")
    L.set_compute_positions(order, xyzq)
    torch.cuda.synchronize()
    assert np.array_equal(xyzq.cpu().numpy(), restate_positions(L, order_h, p.atomStorageSize))
    # per-slot types / indices: an evaluation on device-built arrays equals one on
    # host-uploaded arrays bit for bit (fixed-point forces, pair set, exclusions)
    from helpers import GpuRun
    ref = GpuRun(p)
    ref.build()
    F0, S0, r0, X0 = ref.eval(ALL | nbk.NBK_PAIRLIST, xyzq=xyzq)
    run = GpuRun(p)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    run.nb.set_exclusions_by_atom(L.excl_by_atom)
    run.nb.update_vdw_types_excl_device(L, order, status=status)
    run.nb.build_tile_lists(p, xyzq=xyzq)
    F1, S1, r1, X1 = run.eval(ALL | nbk.NBK_PAIRLIST, xyzq=xyzq)
    assert int(status.item()) == 0
    assert np.array_equal(X0, X1)
    assert r0["energyVdw"] == r1["energyVdw"] and r0["energyElec"] == r1["energyElec"]
    assert run.nb.stat().numExcluded == ref.nb.stat().numExcluded


@pytest.mark.gpu
def test_resident_pipeline_vs_oracle(system):
    """Device sort, positions and types, then tile lists and forces: the atom
    pairs equal the oracle's and the per-atom forces are within tolerance."""
    import torch
    from helpers import GpuRun
    s, p = system
    o = oracle.Oracle(p, PARAMS)
    L = nbk.ResidentLayout(s, p, shuffle_seed=11)
    order = torch.zeros(len(L.ids), dtype=torch.int32, device="cuda")
    L.sort_patch_atoms(order)
    xyzq = torch.zeros((p.atomStorageSize, 4), dtype=torch.float32, device="cuda")
    L.set_compute_positions(order, xyzq)
    run = GpuRun(p)
    run.nb.set_exclusions_by_atom(L.excl_by_atom)
    run.nb.update_vdw_types_excl_device(L, order)
    run.nb.build_tile_lists(p, xyzq=xyzq)
    F, S, res, _ = run.eval(ALL | nbk.NBK_PAIRLIST, xyzq=xyzq)
    slot_ids = restate_slots(L, order.cpu().numpy(), p.atomStorageSize)
    # atom pairs
    tl, ja, ex = run.nb.export_tile_lists()
    mine = nbk.pairs_from_tile_lists(tl, ja, ex, p.atomStorageSize)
    keys, nex = o.pairs()
    n = np.uint64(p.atomStorageSize)

    def atom_pairs(k, ids):
        ids = np.asarray(ids, np.int64)
        i, j = ids[(k // n).astype(np.int64)], ids[(k % n).astype(np.int64)]
        return np.sort(np.minimum(i, j) * (1 << 32) + np.maximum(i, j))

    assert np.array_equal(atom_pairs(mine, slot_ids), atom_pairs(keys, p.atomIndex))
    assert run.nb.stat().numExcluded == nex
    # per-atom forces (the positions differ from the host packing only in the
    # charges' FP32 rounding, far below the tolerance)
    Fo, So, ro = o.forces(1)
    first = {}
    for k, a in enumerate(slot_ids):
        if a >= 0 and a not in first:
            first[a] = k
    atoms = np.arange(s.natoms)
    dev_slot = np.array([first[a] for a in atoms])
    host_slot = p.slotOfAtom[atoms]
    assert rms_rel(F[dev_slot], Fo[host_slot]) < FORCE_RMS_TOL
    assert rms_rel(S[dev_slot], So[host_slot]) < FORCE_RMS_TOL
    assert abs(res["energyVdw"] - ro["energyVdw"]) <= ENERGY_TOL * abs(ro["energyVdw"])


@pytest.mark.gpu
def test_accumulate_forces_to_soa_exact(system):
    """The integrator's FP64 force arrays from the fixed-point sums, the PME
    forces and the bonded arrays: bit for bit the sums a host forms from the
    exported fixed-point forces, in buffer order, at every force level."""
    import torch
    from helpers import GpuRun
    s, p = system
    L = nbk.ResidentLayout(s, p, shuffle_seed=13)
    order = torch.zeros(len(L.ids), dtype=torch.int32, device="cuda")
    L.sort_patch_atoms(order)
    xyzq = torch.zeros((p.atomStorageSize, 4), dtype=torch.float32, device="cuda")
    L.set_compute_positions(order, xyzq)
    run = GpuRun(p)
    run.nb.set_exclusions_by_atom(L.excl_by_atom)
    run.nb.update_vdw_types_excl_device(L, order)
    run.nb.build_tile_lists(p, xyzq=xyzq)
    _, _, _, X = run.eval(ALL | nbk.NBK_PAIRLIST, xyzq=xyzq)
    n = len(L.ids)
    rng = np.random.default_rng(5)
    bond = [rng.normal(size=(3, n)) for _ in range(3)]
    pmef = rng.normal(size=(n, 3)).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    outs = [torch.full((3, n), np.nan, dtype=torch.float64, device="cuda") for _ in range(3)]
    run.nb.accumulate_forces_to_soa(L, order, 2, *outs, f_bond=dev(bond[0]),
                                    f_bond_nbond=dev(bond[1]), f_bond_slow=dev(bond[2]),
                                    f_pme=dev(pmef))
    normal, nbond, slow = (o.cpu().numpy() for o in outs)
    o = order.cpu().numpy()
    slot_of_buf = np.empty(n, dtype=np.int64)
    for q in range(L.numPatches):
        b, nb, k = L.records[q, 1], L.records[q, 2], L.records[q, 3]
        slot_of_buf[b + o[b:b + k]] = nb + np.arange(k)
    fixed = X.astype(np.int64)[:, slot_of_buf].astype(np.float64) * (1.0 / 4294967296.0)
    assert np.array_equal(normal, bond[0])
    assert np.array_equal(nbond, fixed[:3] + bond[1])
    assert np.array_equal(slow, (pmef.T.astype(np.float64) + fixed[3:]) + bond[2])
    # level 0 leaves the other arrays untouched
    keep = [torch.full((3, n), 7.0, dtype=torch.float64, device="cuda") for _ in range(2)]
    run.nb.accumulate_forces_to_soa(L, order, 0, outs[0], *keep)
    assert bool((keep[0] == 7.0).all()) and bool((keep[1] == 7.0).all())
