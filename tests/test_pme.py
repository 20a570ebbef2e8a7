"""PME reciprocal space (nbk_pme_*).

CPU: the FP64 restatement (oracle/pme.py) is pinned to the direct Ewald
reciprocal sum (order 8 on a 64^3 grid, where smooth PME converges to it), its
forces are the gradient of its energy and its virial the strain derivative
(finite differences).
GPU: the product against the restatement on the same FP32 atoms -- energies,
virials and forces -- for B-spline orders 4, 6 and 8, a triclinic cell,
bit-for-bit determinism, the device conversion of positions to fractional
atoms and the self energy.
"""
import numpy as np
import pytest

import nbk
import pme as opme
from helpers import mixed_box, rms_rel, water_box

BETA = 0.2579
QSCALE = float(np.sqrt(332.0636))
# FP32 grid, FFT and interpolation against the FP64 restatement of the same
# algorithm on the same FP32 atoms
PME_ENERGY_TOL = 1e-5
PME_FORCE_RMS_TOL = 1e-5
PME_VIRIAL_TOL = 1e-5


def small_water():
    s = water_box(seed=3, nwater=300, box=21.0)
    a = s.arrays()
    pos = np.asarray(a["pos"], dtype=np.float64).reshape(-1, 3)
    L = np.diag(np.asarray(a["box"], dtype=np.float64))
    atoms = opme.fractional_atoms(pos, a["charge"], L, qscale=QSCALE)
    return atoms, L


def test_oracle_matches_direct_ewald():
    atoms, L = small_water()
    r = atoms[:, :3].astype(np.float64) @ L
    Ed, Fd = opme.ewald_recip_direct(r, atoms[:, 3].astype(np.float64), L, BETA, tol=1e-18)
    E, W, F = opme.pme(atoms, L, (64, 64, 64), 8, BETA)
    assert abs(E - Ed) <= 1e-9 * abs(Ed)
    assert rms_rel(F, Fd) <= 1e-8
    # the usual smooth-PME accuracy at NAMD's default order on the same grid
    E4, _, F4 = opme.pme(atoms, L, (64, 64, 64), 4, BETA)
    assert abs(E4 - Ed) <= 1e-4 * abs(Ed) and rms_rel(F4, Fd) <= 1e-4


def test_oracle_forces_and_virial_are_derivatives():
    atoms, L = small_water()
    K, order = (32, 32, 32), 6
    E, W, F = opme.pme(atoms, L, K, order, BETA)
    R, _ = opme.reciprocal(L)
    for j in (0, 5, 123):
        for d in range(3):
            ap, am = atoms.copy(), atoms.copy()
            dw = 1e-4 * R[:, d]
            ap[j, :3] = (atoms[j, :3].astype(np.float64) + dw).astype(np.float32)
            am[j, :3] = (atoms[j, :3].astype(np.float64) - dw).astype(np.float32)
            step = (ap[j, :3].astype(np.float64) - am[j, :3].astype(np.float64)) @ L
            fd = -(opme.pme(ap, L, K, order, BETA)[0] - opme.pme(am, L, K, order, BETA)[0]) / step[d]
            assert abs(fd - F[j, d]) <= 1e-6 * max(1.0, abs(F[j, d])), (j, d, fd, F[j, d])
    h = 1e-6
    for i in range(3):
        for k in range(3):
            eps = np.zeros((3, 3))
            eps[i, k] = h
            Ep = opme.pme(atoms, L @ (np.eye(3) + eps), K, order, BETA)[0]
            Em = opme.pme(atoms, L @ (np.eye(3) - eps), K, order, BETA)[0]
            assert abs(-(Ep - Em) / (2 * h) - W[i, k]) <= 1e-6 * np.abs(W).max()


def _gpu_case(atoms, L, K, order):
    import torch
    p = nbk.Pme(K, order, BETA)
    d_atoms = torch.from_numpy(np.ascontiguousarray(atoms)).cuda()
    f = torch.zeros((len(atoms), 3), dtype=torch.float32, device="cuda")
    p.compute(d_atoms, len(atoms), L, f)
    E, W = p.energy_virial()
    return p, d_atoms, f.cpu().numpy().astype(np.float64), E, W


def _systems():
    w = water_box()
    a = w.arrays()
    Lw = np.diag(np.asarray(a["box"], dtype=np.float64))
    aw = opme.fractional_atoms(np.asarray(a["pos"]).reshape(-1, 3), a["charge"], Lw, qscale=QSCALE)
    m = mixed_box(natoms=20000)
    b = m.arrays()
    Lm = np.diag(np.asarray(b["box"], dtype=np.float64))
    am = opme.fractional_atoms(np.asarray(b["pos"]).reshape(-1, 3), b["charge"], Lm, qscale=QSCALE)
    # a triclinic cell: the mixed system's atoms in a sheared lattice
    Lt = Lm.copy()
    Lt[1, 0] = 0.2 * Lm[0, 0]
    Lt[2, 0] = -0.1 * Lm[0, 0]
    Lt[2, 1] = 0.15 * Lm[1, 1]
    return {"water9k": (aw, Lw, (48, 48, 48)), "mixed20k": (am, Lm, (60, 60, 60)),
            "triclinic20k": (am, Lt, (60, 64, 60))}


@pytest.mark.gpu
@pytest.mark.parametrize("which,order", [("water9k", 4), ("mixed20k", 4), ("mixed20k", 6),
                                         ("mixed20k", 8), ("triclinic20k", 4)])
def test_gpu_pme_vs_oracle(which, order):
    atoms, L, K = _systems()[which]
    p, _, F, E, W = _gpu_case(atoms, L, K, order)
    Eo, Wo, Fo = opme.pme(atoms, L, K, order, BETA)
    ef, fr = abs(E - Eo) / abs(Eo), rms_rel(F, Fo)
    vr = np.abs(W - Wo).max() / np.abs(Wo).max()
    print(f"{which} order {order}: energy {ef:.2e} force {fr:.2e} virial {vr:.2e}")
    assert ef <= PME_ENERGY_TOL
    assert fr <= PME_FORCE_RMS_TOL
    assert vr <= PME_VIRIAL_TOL


@pytest.mark.gpu
def test_gpu_pme_deterministic():
    atoms, L, K = _systems()["mixed20k"]
    _, _, F1, E1, W1 = _gpu_case(atoms, L, K, 4)
    _, _, F2, E2, W2 = _gpu_case(atoms, L, K, 4)
    assert np.array_equal(F1, F2) and E1 == E2 and np.array_equal(W1, W2)


@pytest.mark.gpu
def test_gpu_pme_atoms_from_positions_and_self_energy():
    import torch
    m = mixed_box(natoms=20000)
    b = m.arrays()
    pos = np.asarray(b["pos"], dtype=np.float64).reshape(-1, 3)
    q = np.asarray(b["charge"], dtype=np.float32)
    L = np.diag(np.asarray(b["box"], dtype=np.float64))
    origin = np.array([-3.0, 1.5, 0.25])
    want = opme.fractional_atoms(pos, q, L, origin=origin, qscale=QSCALE)
    t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    out = torch.zeros((len(pos), 4), dtype=torch.float32, device="cuda")
    nbk.Pme.atoms_from_positions(t(pos[:, 0]), t(pos[:, 1]), t(pos[:, 2]), t(q), QSCALE,
                                 np.concatenate([L.reshape(-1), origin]), out)
    got = out.cpu().numpy()
    assert np.array_equal(got, want)
    p = nbk.Pme((32, 32, 32), 4, BETA)
    se = p.self_energy(out, len(pos))
    assert abs(se - opme.self_energy(want, BETA)) <= 1e-12 * abs(se)


@pytest.mark.gpu
def test_gpu_ewald_total_is_split_independent():
    """The short-range electrostatics with the excluded-pair corrections, the PME
    reciprocal energy and the self energy add up to the periodic Coulomb
    energy of the non-excluded pairs, which does not depend on the Ewald
    coefficient splitting it between the two kernels: two splits must agree.
    This ties the product's short-range slow term, its corrections and its
    PME to the same charges, units and split."""
    import dataclasses
    from helpers import ALL, PARAMS, GpuRun
    s = water_box()
    p = nbk.Packed(s)
    a = s.arrays()
    L = np.diag(np.asarray(a["box"], dtype=np.float64))
    pos = np.asarray(a["pos"], dtype=np.float64).reshape(-1, 3)
    q = p.xyzq[p.slotOfAtom, 3]                      # the short-range path's FP32 charges
    atoms = opme.fractional_atoms(pos, q, L, qscale=1.0)
    import torch
    d_atoms = torch.from_numpy(atoms).cuda()
    force = torch.zeros((len(atoms), 3), dtype=torch.float32, device="cuda")
    totals, scale = [], 0.0
    # splits whose real-space part is converged at the 12 A cutoff
    # (erfc(beta rc) = 5e-9 and 7e-11)
    for beta in (0.34, 0.38):
        params = dataclasses.replace(PARAMS, ewaldcof=beta)
        run = GpuRun(p, params=params)
        run.build()
        _, _, res, _ = run.eval(ALL | nbk.NBK_PAIRLIST | nbk.NBK_CORRECTIONS)
        pm = nbk.Pme((64, 64, 64), 8, beta)
        pm.compute(d_atoms, len(atoms), L, force)
        erec, _ = pm.energy_virial()
        eself = pm.self_energy(d_atoms, len(atoms))
        total = res["energyElec"] + res["energySlow"] + erec + eself
        print(f"beta {beta}: short-range {res['energyElec'] + res['energySlow']:.6f} "
              f"recip {erec:.6f} self {eself:.6f} total {total:.6f}")
        totals.append(total)
        scale = max(scale, abs(eself))
    # the total is a small difference of terms of the self energy's size
    assert abs(totals[0] - totals[1]) <= 1e-7 * scale


def _ref_case(atoms, L, K, order, d_atoms):
    import torch
    import refgpu
    moduli = [opme.b_moduli(k, order) for k in K]
    r = refgpu.RefPme(K, order, BETA, moduli)
    f = torch.zeros((len(atoms), 3), dtype=torch.float32, device="cuda")
    r.compute(d_atoms.data_ptr(), len(atoms), L, f.data_ptr())
    ev = r.energy_virial()
    R = np.linalg.inv(np.asarray(L, np.float64)).T            # rows a*, b*, c*
    F = f.cpu().numpy().astype(np.float64) @ R                # Lattice::scale_force
    xx, xy, xz, yy, yz, zz = ev[1:]
    W = np.array([[xx, xy, xz], [xy, yy, yz], [xz, yz, zz]])
    return r, F, ev[0], W


@pytest.mark.gpu
@pytest.mark.parametrize("which,order", [("water9k", 4), ("mixed20k", 4), ("mixed20k", 6),
                                         ("mixed20k", 8), ("triclinic20k", 4)])
def test_gpu_pme_vs_reference_kernels(which, order):
    """The reference's own PME kernels (spread_charge_v2, scalar_sum,
    gather_force with cuFFT, as CudaPmeOneDevice drives them) on the same FP32
    atoms agree with the product and with the FP64 restatement."""
    import refgpu
    if not refgpu.available():
        pytest.skip("reference kernels not built")
    atoms, L, K = _systems()[which]
    _, d_atoms, F, E, W = _gpu_case(atoms, L, K, order)
    _, Fr, Er, Wr = _ref_case(atoms, L, K, order, d_atoms)
    Eo, Wo, Fo = opme.pme(atoms, L, K, order, BETA)
    for tag, (e, f, w) in {"reference": (Er, Fr, Wr), "product": (E, F, W)}.items():
        ef, fr = abs(e - Eo) / abs(Eo), rms_rel(f, Fo)
        vr = np.abs(w - Wo).max() / np.abs(Wo).max()
        print(f"{which} order {order} {tag} vs oracle: energy {ef:.2e} force {fr:.2e} virial {vr:.2e}")
        assert ef <= PME_ENERGY_TOL and fr <= PME_FORCE_RMS_TOL and vr <= PME_VIRIAL_TOL
    assert abs(E - Er) <= 2 * PME_ENERGY_TOL * abs(Eo)
    assert rms_rel(F, Fr) <= 2 * PME_FORCE_RMS_TOL


@pytest.mark.gpu
def test_gpu_pme_reference_timing():
    """One reciprocal-space evaluation (spread, FFTs, solve with energy and
    virial, gather) of the 92,224-atom mixed system on a 108x108x80 grid,
    order 4: the reference's kernels against the product's, CUDA events on one
    stream with every launch queued while the GPU sleeps."""
    import torch
    import refgpu
    if not refgpu.available():
        pytest.skip("reference kernels not built")
    m = nbk.System(nbk.NBK_SYS_MIXED, 2, 92224, 0.3, box=(108.0, 108.0, 78.0))
    b = m.arrays()
    L = np.diag(np.asarray(b["box"], dtype=np.float64))
    atoms = opme.fractional_atoms(np.asarray(b["pos"]).reshape(-1, 3), b["charge"], L,
                                  qscale=QSCALE)
    K, order, n = (108, 108, 80), 4, len(atoms)
    # the generation order of the system, and the patch order in which NAMD's
    # PME receives atoms (patch by patch, each patch in its bisection order)
    patch_order = np.argsort(nbk.Packed(m).slotOfAtom, kind="stable")
    f = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    p = nbk.Pme(K, order, BETA)
    r = refgpu.RefPme(K, order, BETA, [opme.b_moduli(k, order) for k in K])
    st = torch.cuda.current_stream()
    out = {}
    for tag, idx in (("generation", np.arange(n)), ("patch", patch_order)):
        d_atoms = torch.from_numpy(np.ascontiguousarray(atoms[idx])).cuda()
        calls = {"product": lambda: p.compute(d_atoms, n, L, f, stream=st.cuda_stream),
                 "reference": lambda: r.compute(d_atoms.data_ptr(), n, L, f.data_ptr(),
                                                stream=st.cuda_stream)}
        for name, fn in calls.items():
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            a, z = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda._sleep(50_000_000)
            a.record(st)
            for _ in range(20):
                fn()
            z.record(st)
            torch.cuda.synchronize()
            out[f"{tag}_order_{name}_us"] = round(a.elapsed_time(z) * 1e3 / 20, 2)
    print("pme timing", out)
