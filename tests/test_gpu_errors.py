"""Error paths of the C-ABI (needs a B200 for the handles; every failure is
made on the host). The reference aborts on these (NAMD_die / cudaDie,
src/CudaUtils.C:9-28) or, for a full tile-list buffer, reallocates and
rebuilds (src/CudaTileListKernel.cu:505-509, 1124-1151); here each returns
its status code and leaves the handle usable:
  - NBK_ERR_NOMEM: a device allocation that fails (injected with
    nbk_debug_fail_alloc), in nbk_create, in the set-up calls and in an
    evaluation; after it the same calls succeed and give the results of a
    handle that never failed;
  - NBK_ERR_OVERFLOW: a patch with more tiles than maxTileListLen, or
    maxTileListLen beyond the tile-list format, with tilesSizeExceeded set;
  - NBK_ERR_STATE: calls made out of order.
"""
import ctypes as C

import numpy as np
import pytest

import nbk
from helpers import ALL, PARAMS, water_box

pytestmark = pytest.mark.gpu

OK, ERR_ARG, ERR_STATE, ERR_NOMEM, ERR_OVERFLOW = 0, -1, -3, -4, -5


@pytest.fixture(scope="module")
def system():
    s = water_box(seed=5, nwater=1500, box=36.0)
    return s, nbk.Packed(s)


@pytest.fixture(autouse=True)
def disarm():
    yield
    nbk.dev_lib().nbk_debug_fail_alloc(0)


def _params(lj):
    p = nbk.Params()
    pr = PARAMS
    p.cutoff, p.switchdist, p.pairlistdist, p.ewaldcof = pr.cutoff, pr.switchdist, pr.pairlistdist, pr.ewaldcof
    p.scaling, p.scale14, p.slowScale = pr.scaling, pr.scale14, pr.slowScale
    p.vdwTableDim = lj[0]
    arrs = [np.ascontiguousarray(a, np.float64) for a in lj[1:]]
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    p.ljA, p.ljB, p.ljA14, p.ljB14 = (dp(a) for a in arrs)
    return p, arrs


def _build_raw(nb, packed, max_tiles):
    v = packed.v
    pl = np.float32(PARAMS.pairlistdist)
    return nbk.dev_lib().nbk_build_tile_lists(nb._h, v.numPatches, v.atomStorageSize, max_tiles,
                                              v.lata, v.latb, v.latc,
                                              C.cast(v.patches, C.c_void_p),
                                              packed.xyzq.ctypes.data, 0, float(pl * pl), None)


def _force_raw(nb, packed, flags):
    v = packed.v
    rc = np.float32(PARAMS.cutoff)
    return nbk.dev_lib().nbk_nonbonded_force(nb._h, v.atomStorageSize, flags, v.lata, v.latb,
                                             v.latc, packed.xyzq.ctypes.data, 0, float(rc * rc),
                                             None, None, None, None, None, None)


def _adjoint_raw(nb, packed, dim):
    """nbk_adjoint with valid device buffers, so that only the handle's state decides."""
    import torch
    n = packed.atomStorageSize
    w = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    g = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    gab = torch.zeros(2 * dim * dim, dtype=torch.float64, device="cuda")
    rc = nbk.dev_lib().nbk_adjoint(nb._h, nbk.NBK_SLOW, w.data_ptr(), w.data_ptr(), 0.0, 0.0,
                                   0.0, None, g.data_ptr(), None, gab.data_ptr(), None)
    torch.cuda.synchronize()
    return rc


def _fixed_forces(nb, packed):
    import torch
    X = torch.zeros((6, packed.atomStorageSize), dtype=torch.int64, device="cuda")
    nb.force(packed, ALL, xyzq=packed.xyzq, d_fixed=X)
    ve = nb.virial_energy(ALL)
    return X.cpu().numpy(), (ve.energyVdw, ve.energyElec, ve.energySlow)


def test_create_reports_out_of_memory(system):
    s, p = system
    L = nbk.dev_lib()
    prm, keep = _params(s.lj_table())
    h = C.c_void_p()
    assert L.nbk_debug_fail_alloc(1) == OK
    assert L.nbk_create(0, C.byref(prm), C.byref(h)) == ERR_NOMEM
    assert not h.value, "no handle on failure"
    assert b"out of memory" in L.nbk_last_error()
    assert L.nbk_create(0, C.byref(prm), C.byref(h)) == OK      # the next one allocates
    assert L.nbk_destroy(h) == OK


def test_out_of_memory_in_setup_and_evaluation_is_recoverable(system):
    s, p = system
    L = nbk.dev_lib()
    ref = nbk.Nonbonded(PARAMS, s.lj_table())
    ref.setup(p)
    ref.build_tile_lists(p)
    ref.force(p, ALL | nbk.NBK_PAIRLIST, xyzq=p.xyzq)
    X0, E0 = _fixed_forces(ref, p)

    nb = nbk.Nonbonded(PARAMS, s.lj_table())
    v = p.v
    L.nbk_debug_fail_alloc(1)
    rc = L.nbk_update_computes(nb._h, v.numComputes, C.cast(v.computes, C.c_void_p), None)
    assert rc == ERR_NOMEM, nbk.dev_lib().nbk_last_error()
    nb.setup(p)                                   # allocates normally now
    assert _build_raw(nb, p, v.maxTileListLen) == OK
    # fail each of the first few allocations of the pairlist evaluation in turn
    failed = 0
    for k in range(1, 6):
        L.nbk_debug_fail_alloc(k)
        rc = _force_raw(nb, p, ALL | nbk.NBK_PAIRLIST)
        L.nbk_debug_fail_alloc(0)
        if rc == ERR_NOMEM:
            failed += 1
            assert _build_raw(nb, p, v.maxTileListLen) == OK
        else:
            assert rc == OK
    assert failed >= 1, "no allocation happened in the evaluation"
    assert _build_raw(nb, p, v.maxTileListLen) == OK
    assert _force_raw(nb, p, ALL | nbk.NBK_PAIRLIST) == OK
    X1, E1 = _fixed_forces(nb, p)
    assert np.array_equal(X0, X1) and E0 == E1
    nb.close()
    ref.close()


def test_tile_list_size_limits_overflow(system):
    s, p = system
    L = nbk.dev_lib()
    nb = nbk.Nonbonded(PARAMS, s.lj_table())
    nb.setup(p)
    tiles = (p.patches[:, 0] + 31) // 32
    assert tiles.max() > 1
    st = nbk.TileListStat()
    for bad in (int(tiles.max()) - 1, 65536):
        assert _build_raw(nb, p, bad) == ERR_OVERFLOW
        assert L.nbk_get_tile_list_stat(nb._h, C.byref(st), None) == OK
        assert st.tilesSizeExceeded == 1
    assert _build_raw(nb, p, int(tiles.max())) == OK
    assert L.nbk_get_tile_list_stat(nb._h, C.byref(st), None) == OK
    assert st.tilesSizeExceeded == 0
    assert _force_raw(nb, p, ALL | nbk.NBK_PAIRLIST) == OK
    nb.close()


def test_calls_out_of_order(system):
    s, p = system
    L = nbk.dev_lib()
    v = p.v
    nb = nbk.Nonbonded(PARAMS, s.lj_table())
    # a build needs computes and per-slot data first
    assert _build_raw(nb, p, v.maxTileListLen) == ERR_STATE
    assert L.nbk_update_computes(nb._h, v.numComputes, C.cast(v.computes, C.c_void_p), None) == OK
    assert _build_raw(nb, p, v.maxTileListLen) == ERR_STATE
    nb.setup(p)
    # an evaluation needs tile lists, the first one after a build refines them
    assert _force_raw(nb, p, ALL) == ERR_STATE
    assert _build_raw(nb, p, v.maxTileListLen) == OK
    assert _force_raw(nb, p, ALL) == ERR_STATE
    count = C.c_longlong(0)
    assert L.nbk_autotune(nb._h, ALL, 1, None) == ERR_STATE
    assert _adjoint_raw(nb, p, s.lj_table()[0]) == ERR_STATE       # needs refined lists
    assert _force_raw(nb, p, nbk.NBK_SLOW | nbk.NBK_PAIRLIST) == OK
    # a pair count needs an energy evaluation
    assert L.nbk_get_pair_count(nb._h, C.byref(count), None) == ERR_STATE
    assert _force_raw(nb, p, ALL) == OK
    assert L.nbk_get_pair_count(nb._h, C.byref(count), None) == OK and count.value > 0
    assert _adjoint_raw(nb, p, s.lj_table()[0]) == OK
    nb.close()


def test_batched_handle_refuses_single_system_calls():
    systems = [water_box(seed=40 + k, nwater=n, box=b) for k, (n, b) in
               enumerate(((700, 28.0), (1100, 32.0)))]
    many = nbk.Packed.many(systems)
    L = nbk.dev_lib()
    nb = nbk.Nonbonded(PARAMS, systems[0].lj_table())
    nb.setup(many)
    nb.set_replicas(many)
    nb.build_tile_lists(many)
    nb.force(many, ALL | nbk.NBK_PAIRLIST, xyzq=many.xyzq)
    ve = nbk.VirialEnergy()
    assert L.nbk_reduce_virial_energy(nb._h, ALL, C.byref(ve), 0, None) == ERR_STATE
    assert _adjoint_raw(nb, many, systems[0].lj_table()[0]) == ERR_STATE     # not available with replicas
    nb.close()
