"""Parity on the benchmark's own configuration and step protocol (needs a B200).

The 92,224-atom mixed system in the 108 x 108 x 78 A box, with the
benchmark's trajectory: every frame adds N(0, 0.02 A) to the previous one and
the tile lists are rebuilt every 10 frames. Frame 0 builds and refines the
lists (pairlist step); frames 1..9 are steady steps on the frame-0 lists with
moved atoms, each checked against the FP64 oracle evaluated at that frame's
own positions; frame 10 rebuilds, and its refined pair set must equal the
oracle's bit for bit. That the steady steps find exactly the oracle's pairs
within the cutoff on moved atoms is what the pairlist margin (pairlistdist -
cutoff) guarantees (src/CudaComputeNonbonded.C:1168-1216 rebuilds the lists
before atoms can move farther than that margin allows).
"""
import numpy as np
import pytest

import nbk
import oracle
from helpers import (ALL, ENERGY_TOL, FORCE_RMS_TOL, PARAMS, VIRIAL_TOL, GpuRun, compare,
                     real_slots)

pytestmark = pytest.mark.gpu

NATOMS, BOX, FRAC, SEED, SIGMA = 92224, (108.0, 108.0, 78.0), 0.3, 2, 0.02


def _frames(n):
    s = nbk.System(nbk.NBK_SYS_MIXED, SEED, NATOMS, FRAC, box=BOX)
    p = nbk.Packed(s)
    frames = [p.xyzq.copy()]
    for f in range(1, n):
        s.perturb(SEED * 1000003 + f, SIGMA)   # the benchmark's frame seeds
        p.update_positions()
        frames.append(p.xyzq.copy())
    return s, p, frames


def test_benchmark_trajectory_against_oracle():
    s, p, frames = _frames(11)
    o = oracle.Oracle(p, PARAMS)
    run = GpuRun(p)
    real = real_slots(p)
    fl = ALL | nbk.NBK_CORRECTIONS
    for f, x in enumerate(frames):
        o.xyzq[:] = x
        if f % 10 == 0:
            run.nb.build_tile_lists(p, xyzq=x)
            F, S, res, _ = run.eval(fl | nbk.NBK_PAIRLIST, xyzq=x)
            tl, ja, ex = run.nb.export_tile_lists()
            keys = nbk.pairs_from_tile_lists(tl, ja, ex, p.atomStorageSize)
            ref, nex = o.pairs()
            assert np.array_equal(keys, ref), f"frame {f}: refined pair set differs"
            assert run.nb.stat().numExcluded == nex, f
        else:
            F, S, res, _ = run.eval(fl, xyzq=x)
        Fo, So, ro = o.forces(3)
        err = compare(F, S, res, Fo, So, ro, real)
        print(f"frame {f}: " + " ".join(f"{k}={v:.2e}" for k, v in err.items()))
        assert err["force"] <= FORCE_RMS_TOL and err["slow"] <= FORCE_RMS_TOL, (f, err)
        for k in ("energyVdw", "energyElec", "energySlow"):
            assert err[k] <= ENERGY_TOL, (f, k, err)
        assert err["virial"] <= VIRIAL_TOL and err["virialSlow"] <= VIRIAL_TOL, (f, err)
        assert run.nb.pair_count() == ro["pairs"], f
