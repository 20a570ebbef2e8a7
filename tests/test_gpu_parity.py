"""Parity of the GPU path with the FP64 oracle (needs a B200)."""
import numpy as np
import pytest

import nbk
import oracle
from helpers import (ALL, ENERGY_TOL, FORCE_RMS_TOL, PARAMS, VIRIAL_TOL,
                     GpuRun, compare, mixed_box, real_slots, rms_rel, water_box)

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


def _check_forces(system, corr):
    s, p, o = system
    mode = 3 if corr else 1
    extra = nbk.NBK_CORRECTIONS if corr else 0
    Fo, So, ro = o.forces(mode)
    run = GpuRun(p)
    run.build()
    real = real_slots(p)
    for flags in (ALL | nbk.NBK_PAIRLIST | extra, ALL | extra):
        F, S, res, _ = run.eval(flags)
        err = compare(F, S, res, Fo, So, ro, real)
        print(f"flags={flags} " + " ".join(f"{k}={v:.2e}" for k, v in err.items()))
        assert err["force"] <= FORCE_RMS_TOL and err["slow"] <= FORCE_RMS_TOL, err
        assert err["energyVdw"] <= ENERGY_TOL, err
        assert err["energyElec"] <= ENERGY_TOL and err["energySlow"] <= ENERGY_TOL, err
        assert err["virial"] <= VIRIAL_TOL and err["virialSlow"] <= VIRIAL_TOL, err


@pytest.mark.parametrize("corr", [False, True])
def test_forces_water(water, corr):
    _check_forces(water, corr)


@pytest.mark.parametrize("corr", [False, True])
def test_forces_mixed(mixed, corr):
    _check_forces(mixed, corr)


@pytest.mark.parametrize("beta,cutoff,switch,pl,global_table",
                         [(0.34, 10.0, 8.5, 11.5, True), (0.43, 8.0, 7.0, 9.5, True),
                          (PARAMS.ewaldcof, 12.0, 12.0, 13.5, False)])
def test_forces_other_cutoffs(mixed, beta, cutoff, switch, pl, global_table):
    """Shorter cutoffs with the Ewald coefficients that a PME tolerance of
    1e-6 gives for them, and the benchmark's cutoff without LJ switching
    (switchdist = cutoff), against the oracle with the same parameters: the
    pair set, forces, energies and virials. With the shorter cutoffs the
    precise kernel's slow-term table (136 and 186 rows) is too large for
    shared memory and is read from global memory."""
    import dataclasses
    s, p, _ = mixed
    params = dataclasses.replace(PARAMS, ewaldcof=beta, cutoff=cutoff, switchdist=switch,
                                 pairlistdist=pl)
    T, _ = nbk.slow_table(beta, cutoff, pl)
    assert (T.shape[0] * T.shape[1] * 8 * 8 > 40 * 1024) == global_table
    o = oracle.Oracle(p, params)
    Fo, So, ro = o.forces(3)
    run = GpuRun(p, params=params)
    run.build()
    real = real_slots(p)
    for flags in (ALL | nbk.NBK_PAIRLIST | nbk.NBK_CORRECTIONS, ALL | nbk.NBK_CORRECTIONS):
        F, S, res, _ = run.eval(flags)
        err = compare(F, S, res, Fo, So, ro, real)
        print(f"beta {beta} cutoff {cutoff} flags={flags} " +
              " ".join(f"{k}={v:.2e}" for k, v in err.items()))
        assert err["force"] <= FORCE_RMS_TOL and err["slow"] <= FORCE_RMS_TOL, err
        for k in ("energyVdw", "energyElec", "energySlow"):
            assert err[k] <= ENERGY_TOL, (k, err)
        assert err["virial"] <= VIRIAL_TOL and err["virialSlow"] <= VIRIAL_TOL, err
        assert run.nb.pair_count() == ro["pairs"]
    tl, ja, ex = run.nb.export_tile_lists()
    keys = nbk.pairs_from_tile_lists(tl, ja, ex, p.atomStorageSize)
    ref, _ = o.pairs()
    assert np.array_equal(keys, ref)


def test_pair_count(mixed):
    """The GPU's count of interacting pairs (the benchmark's work unit)
    equals the oracle's."""
    s, p, o = mixed
    _, _, ro = o.forces(1)
    run = GpuRun(p)
    run.build()
    run.eval(ALL | nbk.NBK_PAIRLIST)
    assert run.nb.pair_count() == ro["pairs"]
    run.eval(ALL)
    assert run.nb.pair_count() == ro["pairs"]


def test_deterministic(mixed):
    """Bit-identical forces, energies and virials when the same kind of step
    runs again (pairlist steps and steady-state steps sum their per-tile FP32
    partials in different, fixed orders, so the two kinds agree to rounding)."""
    s, p, o = mixed
    run = GpuRun(p)
    run.build()
    _, _, r1, X1 = run.eval(ALL | nbk.NBK_PAIRLIST | nbk.NBK_CORRECTIONS)
    _, _, r2, X2 = run.eval(ALL | nbk.NBK_CORRECTIONS)
    _, _, r3, X3 = run.eval(ALL | nbk.NBK_CORRECTIONS)
    run.build()
    _, _, r4, X4 = run.eval(ALL | nbk.NBK_PAIRLIST | nbk.NBK_CORRECTIONS)
    assert np.array_equal(X2, X3) and np.array_equal(X1, X4)
    for k in ("energyVdw", "energyElec", "energySlow"):
        assert r2[k] == r3[k] and r1[k] == r4[k]
    assert np.array_equal(r2["virial"], r3["virial"]) and np.array_equal(r1["virial"], r4["virial"])
    real = real_slots(p)
    F1 = X1[:3].T.astype(np.float64)[real]
    F2 = X2[:3].T.astype(np.float64)[real]
    assert rms_rel(F2, F1) <= FORCE_RMS_TOL


def _sparse_case(s):
    p = nbk.Packed(s)
    o = oracle.Oracle(p, PARAMS)
    keys, nex = o.pairs()
    run = GpuRun(p)
    run.build()
    F, S, res, _ = run.eval(ALL | nbk.NBK_PAIRLIST | nbk.NBK_CORRECTIONS)
    tl, ja, ex = run.nb.export_tile_lists()
    mine = nbk.pairs_from_tile_lists(tl, ja, ex, p.atomStorageSize)
    assert np.array_equal(mine, keys)
    assert run.nb.stat().numExcluded == nex
    Fo, So, ro = o.forces(3)
    real = real_slots(p)
    scale = max(np.abs(Fo[real]).max(), np.abs(So[real]).max(), 1e-30)
    assert np.abs(F[real] - Fo[real]).max() <= 1e-5 * scale
    assert np.abs(S[real] - So[real]).max() <= 1e-5 * scale
    for k in ("energyVdw", "energyElec", "energySlow"):
        assert abs(res[k] - ro[k]) <= 1e-6 * max(abs(ro[k]), 1e-12), (k, res[k], ro[k])
    # the steady step on the same (possibly empty) lists
    F2, S2, res2, _ = run.eval(ALL | nbk.NBK_CORRECTIONS)
    assert np.abs(F2[real] - Fo[real]).max() <= 1e-5 * scale
    return len(keys), int(p.patches[:, 0].astype(bool).sum()), len(p.patches)


def test_single_molecule_no_pairs():
    """One water in a 28 A box: its three pairs are excluded and its images
    lie beyond the pairlist distance, so every tile list is empty after the
    refinement and only the excluded-pair corrections act; 6 of the 8 patches
    are empty."""
    npairs, full, total = _sparse_case(nbk.System(nbk.NBK_SYS_WATER, 4, 3, 0.0, box=(28.0, 28.0, 28.0)))
    assert npairs == 0 and full == 2 and total == 8


def test_sparse_system_with_empty_patches():
    """30 waters in a 45 A box: most patches are empty, the lists are ragged."""
    npairs, full, total = _sparse_case(nbk.System(nbk.NBK_SYS_WATER, 5, 90, 0.0, box=(45.0, 45.0, 45.0)))
    assert npairs > 0 and full < total


def test_host_outputs_equal_device_outputs(water):
    """Host force and energy outputs hold exactly the device outputs, both for
    page-locked memory (written by the kernels over PCIe) and for pageable
    memory (copied after them)."""
    import torch
    s, p, _ = water
    n = p.atomStorageSize
    run = GpuRun(p)
    run.build()
    run.eval(ALL | nbk.NBK_PAIRLIST)
    nb = run.nb
    dF = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    dS = torch.zeros_like(dF)
    pinF = torch.full((n, 4), 7.0).pin_memory()
    pinS = torch.full((n, 4), 7.0).pin_memory()
    pageF = np.full((n, 4), 7.0, np.float32)
    pageS = np.full((n, 4), 7.0, np.float32)
    dVE = torch.zeros(31, dtype=torch.float64, device="cuda")
    pinVE = torch.full((31,), 7.0, dtype=torch.float64).pin_memory()
    pageVE = np.full(31, 7.0)
    for hF, hS in ((pinF, pinS), (pageF, pageS)):
        nb.force(p, ALL, xyzq=p.xyzq, d_forces=dF, d_forcesSlow=dS, h_forces=hF, h_forcesSlow=hS)
    nb.virial_energy_to(dVE.data_ptr(), True)
    nb.virial_energy_to(pinVE.data_ptr(), False)
    nb.virial_energy_to(pageVE.ctypes.data, False)
    torch.cuda.synchronize()
    for out, dev in ((pinF.numpy(), dF), (pinS.numpy(), dS), (pageF, dF), (pageS, dS)):
        assert np.array_equal(out, dev.cpu().numpy())
    assert np.abs(dF.cpu().numpy()).max() > 0
    ve = dVE.cpu().numpy()
    assert np.array_equal(pinVE.numpy(), ve) and np.array_equal(pageVE, ve)
    assert ve[18] != 0.0 and not ve[21:].any()


def test_pairlist_and_steady_steps_replay_from_a_cuda_graph(mixed):
    """With the patch layout unchanged, a whole pairlist step (tile-list build,
    refinement, compaction, sort, forces, energy read-out) and a steady step
    are captured in CUDA graphs (no host synchronisation, no allocation) and
    their replays on new positions give exactly the direct calls' results."""
    import torch
    s, p, _ = mixed
    n = p.atomStorageSize
    nb = nbk.Nonbonded(PARAMS, s.lj_table())
    nb.setup(p)
    x = torch.from_numpy(p.xyzq.copy()).cuda()
    dF = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    dS = torch.zeros_like(dF)
    dVE = torch.zeros(31, dtype=torch.float64, device="cuda")
    st = torch.cuda.Stream()

    def pairlist_step(cs):
        nb.build_tile_lists(p, xyzq=x, stream=cs)
        nb.force(p, ALL | nbk.NBK_PAIRLIST, xyzq=x, d_forces=dF, d_forcesSlow=dS, stream=cs)
        nb.virial_energy_to(dVE.data_ptr(), True, stream=cs)

    def steady_step(cs):
        nb.force(p, ALL, xyzq=x, d_forces=dF, d_forcesSlow=dS, stream=cs)
        nb.virial_energy_to(dVE.data_ptr(), True, stream=cs)

    with torch.cuda.stream(st):
        pairlist_step(st.cuda_stream)
        steady_step(st.cuda_stream)
    st.synchronize()
    graphs = []
    for step in (pairlist_step, steady_step):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=st):
            step(torch.cuda.current_stream().cuda_stream)
        graphs.append(g)
    rng = np.random.default_rng(11)
    x0 = x.clone()
    for k in range(2):
        moved = x0.clone()
        moved[:, :3] += torch.from_numpy(rng.normal(0.0, 0.02, (n, 3)).astype(np.float32)).cuda()
        out = []
        for use_graph in (True, False):
            x.copy_(moved)
            torch.cuda.synchronize()
            with torch.cuda.stream(st):
                for g, step in zip(graphs, (pairlist_step, steady_step)):
                    if use_graph:
                        g.replay()
                    else:
                        step(st.cuda_stream)
            st.synchronize()
            out.append((dF.clone(), dS.clone(), dVE.clone()))
        for a, b in zip(out[0], out[1]):
            assert torch.equal(a, b)
        assert out[0][2][18].item() != 0.0
    del graphs


def test_refined_lists_are_sorted_longest_first(mixed):
    """After a pairlist step the compacted tile lists come longest first, and
    their j-tile ranges still partition the compacted j tiles exactly once."""
    s, p, _ = mixed
    run = GpuRun(p)
    run.build()
    run.eval(ALL | nbk.NBK_PAIRLIST)
    tl, ja, _ = run.nb.export_tile_lists()
    lens = tl[:, 2] - tl[:, 1] + 1          # jtileEnd - jtileStart + 1
    assert len(lens) > 0 and (lens >= 1).all()
    assert (np.diff(lens) <= 0).all()
    order = np.argsort(tl[:, 1])
    starts, ends = tl[order, 1], tl[order, 2]
    assert starts[0] == 0 and ends[-1] == len(ja) - 1
    assert (starts[1:] == ends[:-1] + 1).all()
