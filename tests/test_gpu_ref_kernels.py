"""The reference's own CUDA kernels, run beside the product on the same inputs
(needs a B200 and oracle/_ref/libref_nbgpu.so, built from the reference tree
by oracle/ref_gpu/Makefile).

- Pair sets: the refined tile lists of the reference (CudaTileListKernel +
  the pairlist pass of nonbondedForceKernel) hold exactly the oracle's pairs,
  hence exactly the product's; the excluded-pair counts agree.
- Forces, energies, virials: the reference's error against the FP64 oracle
  in its texture-table mode (its choice whenever slow forces are on) and in
  direct math (fast forces only). Table mode interpolates linearly between
  texels with hardware filter weights of 8 fractional bits, a systematic
  per-pair error near 1e-5 that the cancelling electrostatic sums amplify;
  the product's error on the same system is asserted to be smaller.
- Timing: the reference's plain GPU path and the product on the 92,224-atom
  mixed system, steady-state and pairlist steps, and on 64 independent
  replicas (the reference one instance per replica, the product batched),
  CUDA events on each path's stream.
"""
import json

import numpy as np
import pytest

import nbk
import oracle
import refgpu
from helpers import (ALL, PARAMS, GpuRun, compare, mixed_box, real_slots, reference_pairs,
                     rel, rms_rel, unordered_keys, water_box)

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refgpu.available(),
                                 reason="reference kernels not built (oracle/ref_gpu)")]


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


def _ref_run(s, p, do_table=1):
    ref = refgpu.RefGpu(PARAMS, s.lj_table(), do_table=do_table)
    ref.setup(p)
    return ref


def _pairset(system):
    s, p, o = system
    ref = _ref_run(s, p)
    ku, nexcl = reference_pairs(ref, np.ascontiguousarray(p.xyzq), p.atomStorageSize)
    ok, nex = o.pairs()
    assert len(np.unique(ku)) == len(ku), "reference lists a pair twice"
    assert np.array_equal(ku, unordered_keys(ok, p.atomStorageSize))
    assert nexcl == nex
    # the product's lists hold the same pairs
    run = GpuRun(p)
    run.build()
    run.eval(ALL | nbk.NBK_PAIRLIST)
    tl2, ja2, ex2 = run.nb.export_tile_lists()
    mine = nbk.pairs_from_tile_lists(tl2, ja2, ex2, p.atomStorageSize)
    assert np.array_equal(unordered_keys(mine, p.atomStorageSize), ku)
    print(f"pairs {len(ku)} excluded {nexcl}: reference == oracle == product")


def test_ref_pairset_water(water):
    _pairset(water)


def test_ref_pairset_mixed(mixed):
    _pairset(mixed)


def _ref_errors(system, do_table, slow):
    s, p, o = system
    Fo, So, ro = o.forces(1)
    real = real_slots(p)
    ref = _ref_run(s, p, do_table)
    xyzq = np.ascontiguousarray(p.xyzq)
    out = {}
    for pl in (1, 0):
        ref.eval(pl, 1, 1, slow, xyzq)
        F, S, ve = ref.results()
        e = dict(force=rms_rel(F[real, :3].astype(np.float64), Fo[real]),
                 energyVdw=rel(ve[18], ro["energyVdw"]), energyElec=rel(ve[19], ro["energyElec"]),
                 virial=rms_rel(ve[:9].reshape(3, 3), ro["virial"]))
        if slow:
            e.update(slow=rms_rel(S[real, :3].astype(np.float64), So[real]),
                     energySlow=rel(ve[20], ro["energySlow"]),
                     virialSlow=rms_rel(ve[9:18].reshape(3, 3), ro["virialSlow"]))
        out["pairlist" if pl else "steady"] = e
    return out


@pytest.mark.parametrize("which", ["water", "mixed"])
def test_ref_accuracy_table(which, water, mixed):
    """Reference texture-table mode, energy + virial + slow (its production
    configuration). Its error is printed; the product's is asserted at
    1e-5 RMS elsewhere."""
    system = water if which == "water" else mixed
    err = _ref_errors(system, do_table=1, slow=1)
    s, p, o = system
    Fo, So, ro = o.forces(1)
    run = GpuRun(p)
    run.build()
    F, S, res, _ = run.eval(ALL | nbk.NBK_PAIRLIST)
    mine = compare(F, S, res, Fo, So, ro, real_slots(p))
    print(f"product {which}: " + " ".join(f"{k}={v:.2e}" for k, v in mine.items()))
    for step, e in err.items():
        print(f"reference table mode {which} {step}: " + " ".join(f"{k}={v:.2e}" for k, v in e.items()))
        assert e["force"] < 0.2 and e["slow"] < 0.2, e   # harness sanity
        assert mine["force"] < e["force"] and mine["slow"] < e["slow"]


@pytest.mark.parametrize("which", ["water", "mixed"])
def test_ref_accuracy_math(which, water, mixed):
    """Reference direct-math mode (fast forces only: the reference refuses
    direct math when slow forces are on)."""
    system = water if which == "water" else mixed
    err = _ref_errors(system, do_table=0, slow=0)
    for step, e in err.items():
        print(f"reference math mode {which} {step}: " + " ".join(f"{k}={v:.2e}" for k, v in e.items()))
        assert e["force"] < 1e-3, e


def test_ref_plain_path_timing():
    """Steady-state and pairlist eval of the reference plain GPU path and of
    the product on the 92,224-atom mixed system (108 x 108 x 78 A), energy +
    virial + slow forces, positions resident on the device."""
    import torch
    s = nbk.System(nbk.NBK_SYS_MIXED, 11, 92224, 0.3, box=(108.0, 108.0, 78.0))
    p = nbk.Packed(s)
    xyzq = np.ascontiguousarray(p.xyzq)
    K = 200

    def timed(stream, fn, k):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / k

    out = {}
    for do_table in (1, 0):
        slow = 1 if do_table else 0
        ref = _ref_run(s, p, do_table)
        rs = torch.cuda.ExternalStream(ref.stream_ptr)
        ref.eval(1, 1, 1, slow, xyzq)
        ref.sync()
        for _ in range(5):
            ref.eval(0, 1, 1, slow, None)
        key = "table_EVS" if do_table else "math_EV"
        out[f"ref_{key}_steady_ms"] = timed(rs, lambda: ref.eval(0, 1, 1, slow, None), K)
        out[f"ref_{key}_pairlist_ms"] = timed(rs, lambda: ref.eval(1, 1, 1, slow, xyzq), 10)
        del ref

    run = GpuRun(p)
    dx = torch.from_numpy(xyzq).cuda()
    ve_buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    cs = torch.cuda.current_stream()
    for flags, key in ((ALL, "EVS"), (nbk.NBK_ENERGY | nbk.NBK_VIRIAL, "EV")):
        run.nb.build_tile_lists(p, xyzq=dx)
        run.nb.force(p, flags | nbk.NBK_PAIRLIST, xyzq=dx, d_forces=run.dF, d_forcesSlow=run.dS,
                     d_fixed=run.dX)
        for _ in range(5):
            run.nb.force(p, flags, xyzq=dx, d_forces=run.dF, d_forcesSlow=run.dS, d_fixed=run.dX)
        out[f"product_{key}_steady_ms"] = timed(
            cs, lambda: (run.nb.force(p, flags, xyzq=dx, d_forces=run.dF, d_forcesSlow=run.dS,
                                      d_fixed=run.dX),
                         run.nb.virial_energy_to(ve_buf.data_ptr(), True, flags)), K)

        def pl_step():
            run.nb.build_tile_lists(p, xyzq=dx)
            run.nb.force(p, flags | nbk.NBK_PAIRLIST, xyzq=dx, d_forces=run.dF,
                         d_forcesSlow=run.dS, d_fixed=run.dX)
        out[f"product_{key}_pairlist_ms"] = timed(cs, pl_step, 10)
    print("plain-path timing " + json.dumps({k: round(v, 4) for k, v in out.items()}))
    assert all(v > 0 for v in out.values())


def test_ref_kernel_launches_small(mixed):
    """One pairlist and two steady-state evals of each path on the 20,000-atom
    mixed system: reference table mode (E+V+S), reference direct math (E+V),
    product (E+V+S). The fixed launch sequence for kernel profiles."""
    s, p, o = mixed
    xyzq = np.ascontiguousarray(p.xyzq)
    for do_table, slow in ((1, 1), (0, 0)):
        ref = _ref_run(s, p, do_table)
        ref.eval(1, 1, 1, slow, xyzq)
        ref.eval(0, 1, 1, slow, None)
        ref.eval(0, 1, 1, slow, None)
        ref.sync()
        del ref
    run = GpuRun(p)
    run.build()
    for flags in (ALL | nbk.NBK_PAIRLIST, ALL, ALL):
        run.eval(flags)


def test_ref_plain_batch64_timing():
    """64 independent replicas (log-uniform 2,000-40,000 atoms, 0.1 atoms/A^3,
    own seeds; the benchmark's replica set): the reference plain GPU path,
    one reference instance and one launch sequence per replica back to back
    on one stream, against the product's batched handle (all replicas in one
    launch sequence), steady-state energy + virial + slow evaluations with
    positions resident on the device."""
    import torch
    rng = np.random.default_rng(20261203)
    sizes = np.exp(rng.uniform(np.log(2000), np.log(40000), 64)).astype(int)
    systems = [nbk.System(nbk.NBK_SYS_MIXED, 5000 + r, int(n), 0.3) for r, n in enumerate(sizes)]
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    refs = []
    for sy in systems:
        pk = nbk.Packed(sy)
        ref = _ref_run(sy, pk, 1)
        ref.set_stream(sp)
        ref.eval(1, 1, 1, 1, np.ascontiguousarray(pk.xyzq))
        refs.append(ref)
    K = 20

    def timed(fn, k):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(2):
            fn()
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / k

    def ref_round():
        for ref in refs:
            ref.eval(0, 1, 1, 1, None)
    ref_ms = timed(ref_round, K)

    many = nbk.Packed.many(systems)
    nb = nbk.Nonbonded(PARAMS, systems[0].lj_table(), 0)
    nb.setup(many, stream=sp)
    nb.set_replicas(many, stream=sp)
    n = many.atomStorageSize
    with torch.cuda.stream(stream):
        x = torch.from_numpy(many.xyzq.copy()).cuda()
        dF = torch.zeros((n, 4), device="cuda")
        dS = torch.zeros((n, 4), device="cuda")
        dVE = torch.zeros((64, 32), dtype=torch.float64, device="cuda")
    FL = nbk.NBK_ENERGY | nbk.NBK_VIRIAL | nbk.NBK_SLOW
    nb.build_tile_lists(many, xyzq=x, stream=sp)
    nb.force(many, FL | nbk.NBK_PAIRLIST, xyzq=x, d_forces=dF, d_forcesSlow=dS, stream=sp)

    def batch_round():
        nb.force(many, FL, xyzq=x, d_forces=dF, d_forcesSlow=dS, stream=sp)
        nb.virial_energy_batch_to(dVE.data_ptr(), True, stream=sp)
    batch_ms = timed(batch_round, K)
    out = {"replicas": 64, "atoms": int(sizes.sum()), "ref_plain_ms_per_round": round(ref_ms, 4),
           "product_batched_ms_per_round": round(batch_ms, 4),
           "ref_plain_replica_evals_per_s": round(64e3 / ref_ms, 1),
           "product_batched_replica_evals_per_s": round(64e3 / batch_ms, 1),
           "speedup": round(ref_ms / batch_ms, 3)}
    print("batch64 plain-path timing " + json.dumps(out))
    assert ref_ms > 0 and batch_ms > 0
