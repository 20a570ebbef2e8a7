"""Launch-shape autotuner of the force kernel (needs a B200): every shape gives
bit-identical fixed-point forces, energies and virials, and nbk_autotune keeps
one of the shapes it timed."""
import numpy as np
import pytest

import nbk
from helpers import ALL, GpuRun, mixed_box

pytestmark = pytest.mark.gpu


def test_every_launch_shape_gives_identical_results():
    p = nbk.Packed(mixed_box(natoms=20000))
    run = GpuRun(p)
    run.build()
    run.eval(ALL | nbk.NBK_PAIRLIST)
    ref = None
    for b in (4, 5, 6):
        for sp in (1, 2, 4):
            run.nb.set_tuning(ALL, b, sp)
            assert run.nb.tuning(ALL)["ctas_per_sm"] == b
            assert run.nb.tuning(ALL)["warps_per_list"] == sp
            _, _, res, X = run.eval(ALL)
            if ref is None:
                ref = (res, X)
                continue
            assert np.array_equal(X, ref[1]), (b, sp)
            for k in ("energyVdw", "energyElec", "energySlow"):
                assert res[k] == ref[0][k], (b, sp, k)
            assert np.array_equal(res["virial"], ref[0]["virial"])
            assert np.array_equal(res["virialSlow"], ref[0]["virialSlow"])


def test_autotune_keeps_a_timed_shape():
    p = nbk.Packed(mixed_box(natoms=20000))
    run = GpuRun(p)
    run.build()
    _, _, r0, X0 = run.eval(ALL | nbk.NBK_PAIRLIST)
    t = run.nb.autotune(ALL, iterations=3)
    assert t["ctas_per_sm"] in (4, 5, 6) and t["warps_per_list"] in (1, 2, 4) and t["ms"] > 0
    _, _, r1, X1 = run.eval(ALL)
    _, _, r2, X2 = run.eval(ALL)
    assert np.array_equal(X1, X2)
    assert r1["energyVdw"] == r2["energyVdw"]
    print("autotuned shape", t)


def test_launch_sequence_per_register_cap():
    """One pairlist evaluation, then one steady evaluation at 4, 5 and 6 CTAs
    per SM (one warp per tile list) on the 20,000-atom mixed system: the fixed
    launch sequence of the per-register-cap kernel profiles."""
    p = nbk.Packed(mixed_box(natoms=20000))
    run = GpuRun(p)
    run.build()
    run.eval(ALL | nbk.NBK_PAIRLIST)
    for b in (4, 5, 6):
        run.nb.set_tuning(ALL, b, 1)
        run.eval(ALL)
