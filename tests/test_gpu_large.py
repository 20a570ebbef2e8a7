"""Precision study on a 1,066,628-atom system (needs a B200).

The system: 25% seeded random-walk chains + TIP3P-like water at 0.1 atoms/A^3
(a 220.1 A periodic cube), cutoff 12 / switch 10 / pairlist 13.5 A, 1-2/1-3
exclusions, 1-4 pairs scaled 0.833, the exclusion corrections included.
Forces use FP32 pair math folded into 64-bit fixed point; the electrostatic
energies and the slow virial are formed per pair in FP64 and the LJ energy and
fast virial in FP32 (see nbk_nonbonded_force). Force errors are measured
against the FP64 oracle on a seeded 10,000-atom subset; energies and virials
are whole-system quantities, each held to 1e-6 of itself although the
electrostatic totals are ~1e-6 of the sum of |pair energies| here. The table
is printed as one JSON line.
"""
import json

import numpy as np
import pytest

import nbk
import oracle
from helpers import (ALL, ENERGY_TOL, FORCE_RMS_TOL, PARAMS, VIRIAL_TOL, GpuRun, rel, rms_rel)

pytestmark = pytest.mark.gpu

NATOMS, FRAC, SEED, SUBSET = 1066628, 0.25, 4, 10000


def test_large_system_error_table():
    s = nbk.System(nbk.NBK_SYS_MIXED, SEED, NATOMS, FRAC)
    p = nbk.Packed(s)
    o = oracle.Oracle(p, PARAMS)
    Fo, So, ro = o.forces(3)
    rng = np.random.default_rng(20261203)
    atoms = rng.choice(NATOMS, SUBSET, replace=False)
    slots = p.slotOfAtom[atoms]
    run = GpuRun(p)
    run.build()
    table = {"atoms": NATOMS, "box_A": float(s.view().box[0]), "subset_atoms": SUBSET,
             "pairs_in_cutoff": int(ro["pairs"]),
             "energyElec_over_abs_sum": float(abs(ro["energyElec"]) / ro["absElec"])}
    extra = nbk.NBK_CORRECTIONS
    for mode, fl in (("mixed_precision", ALL | extra),):
        for step, f in (("pairlist", fl | nbk.NBK_PAIRLIST), ("steady", fl)):
            F, S, res, _ = run.eval(f)
            e = {
                "force_rms": rms_rel(F[slots], Fo[slots]),
                "slow_rms": rms_rel(S[slots], So[slots]),
                "force_max_atom": float(np.max(np.linalg.norm(F[slots] - Fo[slots], axis=1) /
                                               np.maximum(np.linalg.norm(Fo[slots], axis=1), 1e-12))),
                "energyVdw": rel(res["energyVdw"], ro["energyVdw"]),
                "energyElec": rel(res["energyElec"], ro["energyElec"]),
                "energySlow": rel(res["energySlow"], ro["energySlow"]),
                "energyElec_vs_abs": abs(res["energyElec"] - ro["energyElec"]) / ro["absElec"],
                "energySlow_vs_abs": abs(res["energySlow"] - ro["energySlow"]) / ro["absSlow"],
                "virial": rms_rel(res["virial"], ro["virial"]),
                "virialSlow": rms_rel(res["virialSlow"], ro["virialSlow"]),
            }
            table[f"{mode}_{step}"] = {k: float(f"{v:.3e}") for k, v in e.items()}
            assert e["force_rms"] <= FORCE_RMS_TOL and e["slow_rms"] <= FORCE_RMS_TOL, (mode, e)
            assert e["energyVdw"] <= ENERGY_TOL, (mode, e)
            assert e["energyElec"] <= ENERGY_TOL and e["energySlow"] <= ENERGY_TOL, (mode, e)
            assert e["virial"] <= VIRIAL_TOL and e["virialSlow"] <= VIRIAL_TOL, (mode, e)
    assert run.nb.pair_count() == ro["pairs"]
    print("large-system error table " + json.dumps(table))
