"""The allocation-free corrections entry point, nbk_exclusion_force_noalloc.

It serves callers that cannot call cudaMalloc -- a host framework that owns all
device memory through its own pool, code between captured regions that must not
touch the allocator, runtimes whose device heap is fixed at start-up -- by
keeping its scratch in a static device array instead of allocating. This test
calls it through the C-ABI twice in a row (the second call must not see the
first call's accumulators) and compares each result with what the regular
handle path gives for the same corrections: the difference of one evaluation
with NBK_CORRECTIONS and one without, which isolates the corrections exactly
because the nonbonded part is deterministic.

The file name sorts last so that a run stopping at the first failure has run
every other test; the test also runs alone in a fresh process, where its first
call is the one that looks up the scratch address.
"""
import ctypes as C

import numpy as np
import pytest

import nbk
from helpers import (ALL, ENERGY_TOL, FORCE_RMS_TOL, PARAMS, VIRIAL_TOL, GpuRun, mixed_box,
                     real_slots, rel, rms_rel)


@pytest.mark.gpu
def test_noalloc_corrections_match_handle_path_twice():
    import torch

    s = mixed_box(seed=11, natoms=20000)
    p = nbk.Packed(s)
    n = p.atomStorageSize
    assert n <= 65536
    real = real_slots(p)

    # regular path: corrections = (with) - (without), in fixed point
    run = GpuRun(p)
    run.build()
    run.eval(ALL | nbk.NBK_PAIRLIST)
    _, _, r_without, X_without = run.eval(ALL)
    _, _, r_with, X_with = run.eval(ALL | nbk.NBK_CORRECTIONS)
    dX = (X_with - X_without).astype(np.float64) / nbk.FORCE_FIXED_SCALE
    F_ref, S_ref = dX[:3].T, dX[3:].T

    # inputs of the allocation-free call, in caller-owned device memory
    dim, A, B, A14, B14 = s.lj_table()
    table = np.stack([(A14 - A) * PARAMS.scaling, (B14 - B) * PARAMS.scaling], axis=-1)
    d_table = torch.from_numpy(table.astype(np.float32).reshape(-1)).cuda()
    d_xyzq = torch.from_numpy(p.xyzq.copy()).cuda()
    dF = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    dS = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    dVE = torch.zeros(64, dtype=torch.float64, device="cuda")
    prm = nbk.Params(PARAMS.cutoff, PARAMS.switchdist, PARAMS.pairlistdist, PARAMS.ewaldcof,
                     PARAMS.scaling, PARAMS.scale14, PARAMS.slowScale, dim, None, None, None, None)
    mod = np.ascontiguousarray(p.modified)
    exc = np.ascontiguousarray(p.excluded)
    L = nbk.dev_lib()
    fn = L.nbk_exclusion_force_noalloc
    fn.argtypes = [C.POINTER(nbk.Params), C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int,
                   C.c_void_p, C.c_int, C.c_void_p, nbk.Float3, nbk.Float3, nbk.Float3, C.c_uint,
                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.nbk_noalloc_last_error.restype = C.c_char_p
    v = p.v
    for call in range(2):
        dF.fill_(7.0)   # stale output must be overwritten
        rc = fn(C.byref(prm), d_table.data_ptr(), dim, n, d_xyzq.data_ptr(), len(mod),
                mod.ctypes.data, len(exc), exc.ctypes.data, v.lata, v.latb, v.latc, ALL,
                dF.data_ptr(), dS.data_ptr(), dVE.data_ptr(), None)
        assert rc == 0, L.nbk_noalloc_last_error()
        torch.cuda.synchronize()
        F = dF[:, :3].cpu().numpy().astype(np.float64)
        S = dS[:, :3].cpu().numpy().astype(np.float64)
        ve = nbk.VirialEnergy.from_buffer_copy(dVE.cpu().numpy().tobytes()[:C.sizeof(nbk.VirialEnergy)])
        assert rms_rel(F[real], F_ref[real]) <= FORCE_RMS_TOL, call
        assert rms_rel(S[real], S_ref[real]) <= FORCE_RMS_TOL, call
        for k in ("energyVdw", "energyElec", "energySlow"):
            want = r_with[k] - r_without[k]
            assert abs(getattr(ve, k) - want) <= ENERGY_TOL * max(abs(want), 1.0), (call, k)
        for k in ("virial", "virialSlow"):
            want = r_with[k] - r_without[k]
            got = np.array(getattr(ve, k)).reshape(3, 3)
            assert rms_rel(got, want) <= VIRIAL_TOL, (call, k)

    # sizes beyond the static scratch are refused with a clear error
    rc = fn(C.byref(prm), d_table.data_ptr(), dim, 65536 + 32, d_xyzq.data_ptr(), 0, None, 0,
            None, v.lata, v.latb, v.latc, ALL, dF.data_ptr(), dS.data_ptr(), dVE.data_ptr(), None)
    assert rc == -1 and b"static scratch limit" in L.nbk_noalloc_last_error()
