"""ctypes bindings of the nonbonded path's C-ABI (include/nbk.h) and of the
host-side input preparation (include/nbk_host.h).

This module is the Python face of the library: it loads the in-tree shared
objects (libnbk.so with the sm_100a kernels, libnbk_host.so with the host
preparation) and fails loudly if they are missing. It never computes forces
itself; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

# ---------------------------------------------------------------------------
# POD structs (layouts mirror include/nbk.h)
# ---------------------------------------------------------------------------


class Float3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class Float4(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float), ("w", C.c_float)]


class Int2(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int)]


class ComputeRecord(C.Structure):
    _fields_ = [("patchInd", Int2), ("offsetXYZ", Float3), ("pad", C.c_int)]


class PatchRecord(C.Structure):
    _fields_ = [("numAtoms", C.c_int), ("numFreeAtoms", C.c_int), ("atomStart", C.c_int),
                ("patchID", C.c_int)]


class TileList(C.Structure):
    _fields_ = [("iatomStart", C.c_int), ("jtileStart", C.c_int), ("jtileEnd", C.c_int),
                ("offsetXYZ", Float3), ("patchInd", Int2), ("patchNumList", Int2),
                ("icompute", C.c_int), ("pad", C.c_int)]


class TileListStat(C.Structure):
    _fields_ = [("numTileLists", C.c_int), ("numTileListsGBIS", C.c_int),
                ("numJtiles", C.c_int), ("numExcluded", C.c_int),
                ("patchReadyQueueCount", C.c_int), ("outputOrderIndex", C.c_int),
                ("tilesSizeExceeded", C.c_int)]


class VirialEnergy(C.Structure):
    _fields_ = [("virial", C.c_double * 9), ("virialSlow", C.c_double * 9),
                ("energyVdw", C.c_double), ("energyElec", C.c_double),
                ("energySlow", C.c_double),
                ("energyVdw_s", C.c_double), ("energyElec_s", C.c_double),
                ("energySlow_s", C.c_double),
                ("energyVdw_ti_1", C.c_double), ("energyVdw_ti_2", C.c_double),
                ("energyElec_ti_1", C.c_double), ("energyElec_ti_2", C.c_double),
                ("energySlow_ti_1", C.c_double), ("energySlow_ti_2", C.c_double),
                ("energyGBIS", C.c_double)]


class Exclusion(C.Structure):
    _fields_ = [("i", C.c_int), ("j", C.c_int), ("vdwtypei", C.c_int), ("vdwtypej", C.c_int),
                ("ioffsetXYZ", Float3), ("pswitch", C.c_int)]


class Params(C.Structure):
    _fields_ = [("cutoff", C.c_double), ("switchdist", C.c_double),
                ("pairlistdist", C.c_double), ("ewaldcof", C.c_double),
                ("scaling", C.c_double), ("scale14", C.c_double), ("slowScale", C.c_double),
                ("vdwTableDim", C.c_int),
                ("ljA", C.POINTER(C.c_double)), ("ljB", C.POINTER(C.c_double)),
                ("ljA14", C.POINTER(C.c_double)), ("ljB14", C.POINTER(C.c_double))]


class SystemView(C.Structure):
    _fields_ = [("natoms", C.c_int), ("ntypes", C.c_int), ("numFullExclPairs", C.c_int),
                ("numModPairs", C.c_int), ("numWaters", C.c_int), ("numSolute", C.c_int),
                ("box", C.c_double * 3),
                ("pos", C.POINTER(C.c_double)), ("charge", C.POINTER(C.c_double)),
                ("type", C.POINTER(C.c_int)), ("sigma", C.POINTER(C.c_double)),
                ("epsilon", C.POINTER(C.c_double)), ("fullExcl", C.POINTER(C.c_int)),
                ("modPairs", C.POINTER(C.c_int))]


class PackedView(C.Structure):
    _fields_ = [("natoms", C.c_int), ("numPatches", C.c_int), ("patchGrid", C.c_int * 3),
                ("atomStorageSize", C.c_int), ("maxTileListLen", C.c_int),
                ("numComputes", C.c_int), ("numExclusionWords", C.c_int),
                ("numModified", C.c_int), ("numExcluded", C.c_int),
                ("lata", Float3), ("latb", Float3), ("latc", Float3),
                ("patches", C.POINTER(PatchRecord)), ("computes", C.POINTER(ComputeRecord)),
                ("xyzq", C.POINTER(Float4)), ("vdwTypes", C.POINTER(C.c_int)),
                ("atomIndex", C.POINTER(C.c_int)), ("exclIndexMaxDiff", C.POINTER(Int2)),
                ("exclusionBits", C.POINTER(C.c_uint)), ("modified", C.POINTER(Exclusion)),
                ("excluded", C.POINTER(Exclusion)), ("slotOfAtom", C.POINTER(C.c_int)),
                ("patchCenter", C.POINTER(C.c_double)),
                ("numReplicas", C.c_int), ("replicaOfCompute", C.POINTER(C.c_int)),
                ("replicaSlotStart", C.POINTER(C.c_int)), ("replicaAtomStart", C.POINTER(C.c_int)),
                ("replicaLattice", C.POINTER(Float3))]


NBK_ENERGY, NBK_VIRIAL, NBK_SLOW, NBK_PAIRLIST, NBK_CORRECTIONS = 1, 2, 4, 8, 16
NBK_ENERGY_FP64 = 32
NBK_SYS_WATER, NBK_SYS_MIXED = 0, 1
FORCE_FIXED_SCALE = float(2 ** 32)   # fixed-point units per kcal/mol/A

# ---------------------------------------------------------------------------
# library loading
# ---------------------------------------------------------------------------
_host = None
_dev = None


class NbkError(RuntimeError):
    pass


def _load(name: str) -> C.CDLL:
    path = os.path.join(_HERE, name)
    if not os.path.exists(path):
        raise NbkError(f"{name} is not built (expected at {path}); run __graft_entry__.build()")
    return C.CDLL(path)


def host_lib() -> C.CDLL:
    global _host
    if _host is None:
        lib = _load("libnbk_host.so")
        lib.nbk_host_last_error.restype = C.c_char_p
        lib.nbk_system_generate.argtypes = [C.c_int, C.c_uint64, C.c_int, C.c_double,
                                            C.POINTER(C.c_double), C.POINTER(C.c_void_p)]
        lib.nbk_system_view_get.argtypes = [C.c_void_p, C.POINTER(SystemView)]
        lib.nbk_system_perturb.argtypes = [C.c_void_p, C.c_uint64, C.c_double]
        lib.nbk_system_free.argtypes = [C.c_void_p]
        lib.nbk_lj_table.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                     C.c_int] + [C.POINTER(C.c_double)] * 4
        lib.nbk_pack.argtypes = [C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_void_p)]
        lib.nbk_packed_view_get.argtypes = [C.c_void_p, C.POINTER(PackedView)]
        lib.nbk_pack_update_positions.argtypes = [C.c_void_p, C.c_void_p]
        lib.nbk_lj_param_grad.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.nbk_pack_many.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_double, C.c_double,
                                      C.POINTER(C.c_void_p)]
        lib.nbk_packed_free.argtypes = [C.c_void_p]
        _host = lib
    return _host


def _hcheck(rc: int, what: str):
    if rc != 0:
        msg = host_lib().nbk_host_last_error().decode()
        raise NbkError(f"{what} failed ({rc}): {msg}")


def _arr(ptr, n, dtype):
    if n == 0 or not ptr:
        return np.zeros(0, dtype=dtype)
    buf = C.cast(ptr, C.POINTER(C.c_char * (n * np.dtype(dtype).itemsize))).contents
    return np.frombuffer(buf, dtype=dtype, count=n)


# ---------------------------------------------------------------------------
# synthetic systems and packing
# ---------------------------------------------------------------------------
@dataclass
class NonbondedParams:
    cutoff: float = 12.0
    switchdist: float = 10.0
    pairlistdist: float = 13.5
    ewaldcof: float = 0.2579
    scaling: float = 1.0
    dielectric: float = 1.0
    scale14: float = 0.833
    slowScale: float = 1.0


class System:
    """A seeded synthetic system in global atom order (owned by libnbk_host)."""

    def __init__(self, kind: int, seed: int, natoms: int, solute_frac: float = 0.3, box=None):
        lib = host_lib()
        h = C.c_void_p()
        b = (C.c_double * 3)(*(box if box is not None else (0.0, 0.0, 0.0)))
        _hcheck(lib.nbk_system_generate(kind, seed, natoms, solute_frac, b, C.byref(h)),
                "nbk_system_generate")
        self._h = h
        self.kind = kind
        self.seed = seed

    def __del__(self):
        if getattr(self, "_h", None) and _host is not None:
            _host.nbk_system_free(self._h)
            self._h = None

    def view(self) -> SystemView:
        v = SystemView()
        _hcheck(host_lib().nbk_system_view_get(self._h, C.byref(v)), "nbk_system_view_get")
        return v

    @property
    def natoms(self):
        return self.view().natoms

    def arrays(self):
        v = self.view()
        n, nt = v.natoms, v.ntypes
        return dict(
            pos=_arr(v.pos, 3 * n, np.float64).reshape(n, 3).copy(),
            charge=_arr(v.charge, n, np.float64).copy(),
            type=_arr(v.type, n, np.int32).copy(),
            sigma=_arr(v.sigma, nt, np.float64).copy(),
            epsilon=_arr(v.epsilon, nt, np.float64).copy(),
            fullExcl=_arr(v.fullExcl, 2 * v.numFullExclPairs, np.int32).reshape(-1, 2).copy(),
            modPairs=_arr(v.modPairs, 2 * v.numModPairs, np.int32).reshape(-1, 2).copy(),
            box=np.array(list(v.box)),
            numWaters=v.numWaters, numSolute=v.numSolute)

    def perturb(self, seed: int, sigma: float):
        _hcheck(host_lib().nbk_system_perturb(self._h, seed, sigma), "nbk_system_perturb")

    def lj_table(self, geometric=False):
        v = self.view()
        nt = v.ntypes
        A, B, A14, B14 = (np.zeros(nt * nt) for _ in range(4))
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        _hcheck(host_lib().nbk_lj_table(nt, v.sigma, v.epsilon, int(geometric), dp(A), dp(B),
                                        dp(A14), dp(B14)), "nbk_lj_table")
        return nt, A, B, A14, B14


def lj_param_grad(sigma, epsilon, gA, gB, scaling=1.0, geometric=False):
    """Per-type (dL/dsigma, dL/depsilon) from gradients w.r.t. the scaled LJ
    table entries (nbk_lj_param_grad)."""
    nt = len(sigma)
    sg = np.ascontiguousarray(sigma, dtype=np.float64)
    ep = np.ascontiguousarray(epsilon, dtype=np.float64)
    a = np.ascontiguousarray(gA, dtype=np.float64).reshape(-1)
    b = np.ascontiguousarray(gB, dtype=np.float64).reshape(-1)
    gs, ge = np.zeros(nt), np.zeros(nt)
    _hcheck(host_lib().nbk_lj_param_grad(nt, sg.ctypes.data, ep.ctypes.data, int(geometric),
                                         scaling, a.ctypes.data, b.ctypes.data, gs.ctypes.data,
                                         ge.ctypes.data), "nbk_lj_param_grad")
    return gs, ge


class Packed:
    """Host mirror of CudaComputeNonbonded's inputs for one system, or for
    several independent systems (replicas) concatenated (Packed.many)."""

    def __init__(self, system: System, patch_dim: float = 13.5, coulomb_scaling: float = 1.0,
                 _handle=None, _systems=None):
        lib = host_lib()
        if _handle is None:
            h = C.c_void_p()
            _hcheck(lib.nbk_pack(system._h, patch_dim, coulomb_scaling, C.byref(h)), "nbk_pack")
            self.systems = [system]
            self.coulomb_scaling = coulomb_scaling
        else:
            h = _handle
            self.systems = list(_systems)
        self._h = h
        self.system = self.systems[0]
        self._refresh()

    @classmethod
    def many(cls, systems, patch_dim: float = 13.5, coulomb_scaling: float = 1.0):
        arr = (C.c_void_p * len(systems))(*[x._h for x in systems])
        h = C.c_void_p()
        _hcheck(host_lib().nbk_pack_many(arr, len(systems), patch_dim, coulomb_scaling,
                                         C.byref(h)), "nbk_pack_many")
        out = cls(None, _handle=h, _systems=systems)
        out.coulomb_scaling = coulomb_scaling
        return out

    def __del__(self):
        if getattr(self, "_h", None) and _host is not None:
            _host.nbk_packed_free(self._h)
            self._h = None

    def _refresh(self):
        v = PackedView()
        _hcheck(host_lib().nbk_packed_view_get(self._h, C.byref(v)), "nbk_packed_view_get")
        self.v = v
        n = v.atomStorageSize
        self.atomStorageSize = n
        self.numPatches = v.numPatches
        self.numComputes = v.numComputes
        self.maxTileListLen = v.maxTileListLen
        self.lattice = np.array([[v.lata.x, v.lata.y, v.lata.z], [v.latb.x, v.latb.y, v.latb.z],
                                 [v.latc.x, v.latc.y, v.latc.z]], dtype=np.float32)
        self.xyzq = _arr(v.xyzq, 4 * n, np.float32).reshape(n, 4)
        self.vdwTypes = _arr(v.vdwTypes, n, np.int32)
        self.atomIndex = _arr(v.atomIndex, n, np.int32)
        self.exclIndexMaxDiff = _arr(v.exclIndexMaxDiff, 2 * n, np.int32).reshape(n, 2)
        self.exclusionBits = _arr(v.exclusionBits, v.numExclusionWords, np.uint32)
        self.patches = _arr(v.patches, 4 * v.numPatches, np.int32).reshape(-1, 4)
        comp = _arr(v.computes, 6 * v.numComputes, np.int32).reshape(-1, 6)
        self.computes = comp                                 # raw nbk_compute_record words
        self.computes_patch = comp[:, :2]
        self.computes_offset = comp[:, 2:5].view(np.float32)
        self.slotOfAtom = _arr(v.slotOfAtom, v.natoms, np.int32)
        self.patchCenter = _arr(v.patchCenter, 3 * v.numPatches, np.float64).reshape(-1, 3)
        ex_dt = np.dtype([("i", np.int32), ("j", np.int32), ("ti", np.int32), ("tj", np.int32),
                          ("off", np.float32, 3), ("pswitch", np.int32)])
        self.modified = _arr(v.modified, v.numModified * 32, np.uint8).view(ex_dt)
        self.excluded = _arr(v.excluded, v.numExcluded * 32, np.uint8).view(ex_dt)
        self.numReplicas = v.numReplicas
        self.replicaOfCompute = _arr(v.replicaOfCompute, v.numComputes, np.int32)
        self.replicaSlotStart = _arr(v.replicaSlotStart, v.numReplicas + 1, np.int32)
        self.replicaAtomStart = _arr(v.replicaAtomStart, v.numReplicas + 1, np.int32)
        self.replicaLattice = _arr(v.replicaLattice, 9 * v.numReplicas, np.float32).reshape(-1, 3, 3)

    def update_positions(self):
        _hcheck(host_lib().nbk_pack_update_positions(self._h, self.system._h),
                "nbk_pack_update_positions")
        self._refresh()


# ---------------------------------------------------------------------------
# device path (libnbk.so)
# ---------------------------------------------------------------------------
class TileExcl(C.Structure):
    _fields_ = [("excl", C.c_uint * 32)]


def dev_lib() -> C.CDLL:
    global _dev
    if _dev is None:
        lib = _load("libnbk.so")
        vp, i, u, f = C.c_void_p, C.c_int, C.c_uint, C.c_float
        lib.nbk_last_error.restype = C.c_char_p
        lib.nbk_create.argtypes = [i, C.POINTER(Params), C.POINTER(vp)]
        lib.nbk_destroy.argtypes = [vp]
        lib.nbk_update_computes.argtypes = [vp, i, vp, vp]
        lib.nbk_bind_exclusions.argtypes = [vp, i, vp]
        lib.nbk_update_vdw_types_excl.argtypes = [vp, i, vp, vp, vp, vp]
        lib.nbk_set_exclusion_tuples.argtypes = [vp, i, vp, i, vp, vp]
        lib.nbk_build_tile_lists.argtypes = [vp, i, i, i, Float3, Float3, Float3, vp, vp, i, f, vp]
        lib.nbk_nonbonded_force.argtypes = [vp, i, u, Float3, Float3, Float3, vp, i, f,
                                            vp, vp, vp, vp, vp, vp]
        lib.nbk_reduce_virial_energy.argtypes = [vp, u, C.POINTER(VirialEnergy), i, vp]
        lib.nbk_get_tile_list_stat.argtypes = [vp, C.POINTER(TileListStat), vp]
        lib.nbk_export_tile_lists.argtypes = [vp, C.POINTER(i), C.POINTER(i), vp, vp, vp, vp]
        lib.nbk_set_kernel_timing.argtypes = [vp, i]
        lib.nbk_autotune.argtypes = [vp, u, i, vp]
        lib.nbk_get_tuning.argtypes = [vp, u, C.POINTER(i), C.POINTER(i), C.POINTER(C.c_float)]
        lib.nbk_set_tuning.argtypes = [vp, u, i, i]
        lib.nbk_get_kernel_times.argtypes = [vp, C.POINTER(C.c_float), i, C.POINTER(i)]
        lib.nbk_launch_count.restype = C.c_longlong
        lib.nbk_launch_count.argtypes = [vp]
        lib.nbk_get_pair_count.argtypes = [vp, C.POINTER(C.c_longlong), vp]
        lib.nbk_measure_fp32_peak.argtypes = [i, C.POINTER(C.c_double)]
        lib.nbk_measure_fp64_peak.argtypes = [i, C.POINTER(C.c_double)]
        lib.nbk_debug_fail_alloc.argtypes = [i]
        lib.nbk_get_precise_times.argtypes = [vp, C.POINTER(C.c_float), i, C.POINTER(i)]
        lib.nbk_slow_table.argtypes = [C.c_double, C.c_double, C.c_double, vp, i,
                                       C.POINTER(C.c_double)]
        lib.nbk_set_replicas.argtypes = [vp, i, vp, vp, vp, vp, vp, vp, vp, vp]
        lib.nbk_adjoint.argtypes = [vp, u, vp, vp, C.c_double, C.c_double, C.c_double, vp, vp, vp,
                                    vp, vp]
        lib.nbk_reduce_virial_energy_batch.argtypes = [vp, u, vp, i, vp]
        lib.nbk_get_pair_counts.argtypes = [vp, C.POINTER(C.c_longlong), i, vp]
        lib.nbk_sort_patch_atoms.argtypes = [i, vp, i, vp, vp, vp, vp, vp, vp, vp]
        lib.nbk_set_compute_positions.argtypes = [i, vp, vp, C.POINTER(C.c_double), vp,
                                                  C.c_double, vp, vp, vp, vp, vp, vp]
        lib.nbk_set_exclusions_by_atom.argtypes = [vp, i, vp]
        lib.nbk_update_vdw_types_excl_device.argtypes = [vp, i, i, vp, vp, vp, vp, vp, vp]
        lib.nbk_accumulate_forces_to_soa.argtypes = [vp, i, i, vp, vp, vp, vp, vp, i, vp] + [vp] * 9 + [vp]
        dp = C.POINTER(C.c_double)
        lib.nbk_pme_create.argtypes = [i, C.POINTER(PmeGrid), C.c_double, C.POINTER(vp)]
        lib.nbk_pme_destroy.argtypes = [vp]
        lib.nbk_pme_atoms_from_positions.argtypes = [i, vp, vp, vp, vp, C.c_double, dp, vp, vp]
        lib.nbk_pme_spread_charge.argtypes = [vp, i, vp, vp]
        lib.nbk_pme_solve.argtypes = [vp, dp, u, vp]
        lib.nbk_pme_gather_force.argtypes = [vp, i, vp, dp, vp, vp]
        lib.nbk_pme_get_energy_virial.argtypes = [vp, dp, dp, vp]
        lib.nbk_pme_self_energy.argtypes = [vp, i, vp, dp, vp]
        _dev = lib
    return _dev


class PmeGrid(C.Structure):
    _fields_ = [("K1", C.c_int), ("K2", C.c_int), ("K3", C.c_int), ("order", C.c_int)]


def _dcheck(rc: int, what: str):
    if rc != 0:
        raise NbkError(f"{what} failed ({rc}): {dev_lib().nbk_last_error().decode()}")


def _f3(v):
    return Float3(float(v[0]), float(v[1]), float(v[2]))


def _ptr(a):
    """Address of a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


class Nonbonded:
    """One handle of the B200 nonbonded path: CudaTileListKernel +
    CudaComputeNonbondedKernel + CudaNonbondedTables for one GPU."""

    def __init__(self, params: NonbondedParams, lj, device: int = 0):
        dim, A, B, A14, B14 = lj
        self._lj = [np.ascontiguousarray(x, dtype=np.float64) for x in (A, B, A14, B14)]
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        p = Params(params.cutoff, params.switchdist, params.pairlistdist, params.ewaldcof,
                   params.scaling,
                   params.scale14, params.slowScale, dim, *(dp(a) for a in self._lj))
        self.params = params
        self.device = device
        h = C.c_void_p()
        _dcheck(dev_lib().nbk_create(device, C.byref(p), C.byref(h)), "nbk_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and _dev is not None:
            _dev.nbk_destroy(self._h)
            self._h = None

    __del__ = close

    # -- set-up -------------------------------------------------------------
    def setup(self, packed: Packed, stream=None):
        """Uploads computes, exclusions, per-slot data and correction tuples."""
        L = dev_lib()
        v = packed.v
        _dcheck(L.nbk_update_computes(self._h, v.numComputes, C.cast(v.computes, C.c_void_p),
                                      stream), "nbk_update_computes")
        _dcheck(L.nbk_bind_exclusions(self._h, v.numExclusionWords,
                                      C.cast(v.exclusionBits, C.c_void_p)), "nbk_bind_exclusions")
        _dcheck(L.nbk_update_vdw_types_excl(self._h, v.atomStorageSize,
                                            C.cast(v.vdwTypes, C.c_void_p),
                                            C.cast(v.exclIndexMaxDiff, C.c_void_p),
                                            C.cast(v.atomIndex, C.c_void_p), stream),
                "nbk_update_vdw_types_excl")
        _dcheck(L.nbk_set_exclusion_tuples(self._h, v.numModified, C.cast(v.modified, C.c_void_p),
                                           v.numExcluded, C.cast(v.excluded, C.c_void_p), stream),
                "nbk_set_exclusion_tuples")
        self.packed = packed

    def set_replicas(self, packed: Packed, stream=None):
        """Batched mode: every replica of a Packed.many layout with its own
        lattice and LJ tables (call after setup)."""
        tabs = [x.lj_table() for x in packed.systems]
        dims = {t[0] for t in tabs}
        if len(dims) != 1:
            raise NbkError("replicas must share the number of LJ types")
        cat = [np.ascontiguousarray(np.concatenate([t[k] for t in tabs])) for k in (1, 2, 3, 4)]
        self._rep_lj = cat
        lat = np.ascontiguousarray(packed.replicaLattice.reshape(-1, 3), dtype=np.float32)
        self._rep_lat = lat
        roc = np.ascontiguousarray(packed.replicaOfCompute, dtype=np.int32)
        rss = np.ascontiguousarray(packed.replicaSlotStart, dtype=np.int32)
        self._rep_idx = (roc, rss)
        _dcheck(dev_lib().nbk_set_replicas(self._h, packed.numReplicas, roc.ctypes.data,
                                           rss.ctypes.data, lat.ctypes.data,
                                           *(a.ctypes.data for a in cat), stream),
                "nbk_set_replicas")
        self.numReplicas = packed.numReplicas

    def adjoint(self, wF, wS, cV, cE, cS, gradXQ, gradAB, type_mask=None, grad_fixed=None,
                slow=True, stream=None):
        """Gradient of sum wF.F + sum wS.Fslow + cV E_vdw + cE E_elec + cS E_slow
        (nbk_adjoint). wF, wS, gradXQ: device float4[n]; gradAB: device double[2*dim*dim]."""
        mask = None
        if type_mask is not None:
            mask = np.ascontiguousarray(type_mask, dtype=np.int32)
        _dcheck(dev_lib().nbk_adjoint(self._h, NBK_SLOW if slow else 0, _ptr(wF), _ptr(wS),
                                      cV, cE, cS, None if mask is None else mask.ctypes.data,
                                      _ptr(gradXQ), _ptr(grad_fixed), _ptr(gradAB), stream),
                "nbk_adjoint")

    def virial_energy_batch(self, stream=None):
        n = self.numReplicas
        arr = (VirialEnergy * n)()
        _dcheck(dev_lib().nbk_reduce_virial_energy_batch(self._h, NBK_ENERGY | NBK_VIRIAL | NBK_SLOW,
                                                         C.cast(arr, C.c_void_p), 0, stream),
                "nbk_reduce_virial_energy_batch")
        import torch
        torch.cuda.synchronize(self.device)
        return list(arr)

    def virial_energy_batch_to(self, ptr: int, on_device: bool, stream=None):
        _dcheck(dev_lib().nbk_reduce_virial_energy_batch(self._h, NBK_ENERGY | NBK_VIRIAL | NBK_SLOW,
                                                         ptr, int(on_device), stream),
                "nbk_reduce_virial_energy_batch")

    def pair_counts(self, stream=None):
        n = getattr(self, "numReplicas", 1)
        arr = (C.c_longlong * n)()
        _dcheck(dev_lib().nbk_get_pair_counts(self._h, arr, n, stream), "nbk_get_pair_counts")
        return np.array(arr[:], dtype=np.int64)

    def build_tile_lists(self, packed: Packed, xyzq=None, stream=None):
        """xyzq: None (host copy of packed.xyzq) or a device tensor."""
        v = packed.v
        on_dev = xyzq is not None and not isinstance(xyzq, np.ndarray)
        src = _ptr(xyzq) if xyzq is not None else packed.xyzq.ctypes.data
        pl = np.float32(self.params.pairlistdist)
        _dcheck(dev_lib().nbk_build_tile_lists(self._h, v.numPatches, v.atomStorageSize,
                                               v.maxTileListLen, v.lata, v.latb, v.latc,
                                               C.cast(v.patches, C.c_void_p), src, int(on_dev),
                                               float(pl * pl), stream), "nbk_build_tile_lists")

    def force(self, packed: Packed, flags: int, xyzq=None, d_forces=None, d_forcesSlow=None,
              h_forces=None, h_forcesSlow=None, d_fixed=None, stream=None):
        v = packed.v
        on_dev = xyzq is not None and not isinstance(xyzq, np.ndarray)
        src = _ptr(xyzq)
        rc = np.float32(self.params.cutoff)
        _dcheck(dev_lib().nbk_nonbonded_force(self._h, v.atomStorageSize, flags, v.lata, v.latb,
                                              v.latc, src, int(on_dev), float(rc * rc),
                                              _ptr(d_forces), _ptr(d_forcesSlow), _ptr(h_forces),
                                              _ptr(h_forcesSlow), _ptr(d_fixed), stream),
                "nbk_nonbonded_force")

    def virial_energy(self, flags=NBK_ENERGY | NBK_VIRIAL | NBK_SLOW, stream=None,
                      sync=True) -> VirialEnergy:
        ve = VirialEnergy()
        _dcheck(dev_lib().nbk_reduce_virial_energy(self._h, flags, C.byref(ve), 0, stream),
                "nbk_reduce_virial_energy")
        if sync:
            import torch
            torch.cuda.synchronize(self.device)
        return ve

    def virial_energy_to(self, ptr: int, on_device: bool, flags=NBK_ENERGY | NBK_VIRIAL | NBK_SLOW,
                         stream=None):
        """Writes the VirialEnergy record to a raw device or (pinned) host address."""
        _dcheck(dev_lib().nbk_reduce_virial_energy(self._h, flags,
                                                   C.cast(C.c_void_p(ptr), C.POINTER(VirialEnergy)),
                                                   int(on_device), stream),
                "nbk_reduce_virial_energy")

    def stat(self, stream=None) -> TileListStat:
        s = TileListStat()
        _dcheck(dev_lib().nbk_get_tile_list_stat(self._h, C.byref(s), stream),
                "nbk_get_tile_list_stat")
        return s

    def set_kernel_timing(self, enable: bool):
        _dcheck(dev_lib().nbk_set_kernel_timing(self._h, int(enable)), "nbk_set_kernel_timing")

    def _times(self, fn):
        n = C.c_int(0)
        f = getattr(dev_lib(), fn)
        _dcheck(f(self._h, None, 0, C.byref(n)), fn)
        ms = (C.c_float * max(n.value, 1))()
        _dcheck(f(self._h, ms, n.value, C.byref(n)), fn)
        return np.array(ms[:n.value], dtype=np.float64)

    def kernel_times(self):
        """Per recorded evaluation: the force kernel (with the pairlist work
        before it on pairlist evaluations), ms."""
        return self._times("nbk_get_kernel_times")

    def precise_times(self):
        """Per recorded evaluation: the precise energy / virial kernel, ms."""
        return self._times("nbk_get_precise_times")

    def launch_count(self) -> int:
        return int(dev_lib().nbk_launch_count(self._h))

    def pair_count(self, stream=None) -> int:
        n = C.c_longlong(0)
        _dcheck(dev_lib().nbk_get_pair_count(self._h, C.byref(n), stream), "nbk_get_pair_count")
        return int(n.value)

    def autotune(self, flags=NBK_ENERGY | NBK_VIRIAL | NBK_SLOW, iterations=5, stream=None):
        """Times the force kernel's launch shapes on the current refined lists and
        keeps the fastest for these flags (nbk_autotune); returns the choice."""
        _dcheck(dev_lib().nbk_autotune(self._h, flags, iterations, stream), "nbk_autotune")
        return self.tuning(flags)

    def set_tuning(self, flags, ctas_per_sm, warps_per_list):
        """Pins the force kernel's launch shape for these flags (nbk_set_tuning)."""
        _dcheck(dev_lib().nbk_set_tuning(self._h, flags, ctas_per_sm, warps_per_list),
                "nbk_set_tuning")

    def tuning(self, flags=NBK_ENERGY | NBK_VIRIAL | NBK_SLOW):
        """(CTAs per SM, warps per tile list, ms per force launch) for these flags."""
        b, sp, ms = C.c_int(0), C.c_int(0), C.c_float(0)
        _dcheck(dev_lib().nbk_get_tuning(self._h, flags, C.byref(b), C.byref(sp), C.byref(ms)),
                "nbk_get_tuning")
        return {"ctas_per_sm": b.value, "warps_per_list": sp.value, "ms": ms.value}

    # -- GPU-resident input marshaling --------------------------------------
    def set_exclusions_by_atom(self, excl_by_atom):
        """(maxdiff, base) per global atom id, int32 [natoms, 2] (host)."""
        a = np.ascontiguousarray(excl_by_atom, dtype=np.int32)
        _dcheck(dev_lib().nbk_set_exclusions_by_atom(self._h, len(a), a.ctypes.data),
                "nbk_set_exclusions_by_atom")

    def update_vdw_types_excl_device(self, layout, sort_order, status=None, stream=None):
        """Per-slot vdW types / atom indices / exclusion indices from the
        device-resident per-atom arrays of a ResidentLayout."""
        d = layout.dev
        _dcheck(dev_lib().nbk_update_vdw_types_excl_device(
            self._h, layout.numPatches, layout.atomStorageSize, _ptr(d["records"]),
            _ptr(d["vdw"]), _ptr(d["id"]), _ptr(sort_order), _ptr(status), stream),
            "nbk_update_vdw_types_excl_device")

    def accumulate_forces_to_soa(self, layout, sort_order, max_force_number, normal, nbond=None,
                                 slow=None, f_bond=None, f_bond_nbond=None, f_bond_slow=None,
                                 f_pme=None, stream=None):
        """Integrator FP64 force arrays (buffer order) from the last evaluation's
        fixed-point sums: normal, nbond, slow are [3, natoms] float64 tensors;
        f_bond* are [3, natoms] float64 (or None), f_pme [natoms, 3] float32."""
        d = layout.dev
        rows = lambda t: [None] * 3 if t is None else [t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr()]
        fs = 0
        for t in (f_bond, f_bond_nbond, f_bond_slow):
            if t is not None:
                fs = int(t.stride(0))
        _dcheck(dev_lib().nbk_accumulate_forces_to_soa(
            self._h, int(max_force_number), layout.numPatches, _ptr(d["records"]), _ptr(sort_order),
            _ptr(f_bond), _ptr(f_bond_nbond), _ptr(f_bond_slow), fs, _ptr(f_pme),
            *rows(normal), *rows(nbond), *rows(slow), stream), "nbk_accumulate_forces_to_soa")

    def export_tile_lists(self, stream=None):
        nl, nj = C.c_int(0), C.c_int(0)
        L = dev_lib()
        _dcheck(L.nbk_export_tile_lists(self._h, C.byref(nl), C.byref(nj), None, None, None,
                                        stream), "nbk_export_tile_lists")
        tl = np.zeros((max(nl.value, 1), 12), dtype=np.int32)
        ja = np.zeros(max(nj.value, 1), dtype=np.int32)
        ex = np.zeros((max(nj.value, 1), 32), dtype=np.uint32)
        _dcheck(L.nbk_export_tile_lists(self._h, C.byref(nl), C.byref(nj), tl.ctypes.data,
                                        ja.ctypes.data, ex.ctypes.data, stream),
                "nbk_export_tile_lists")
        return tl[:nl.value], ja[:nj.value], ex[:nj.value]


SLOW_TABLE_ROW = 6  # doubles per row of nbk_slow_table (degree-5 polynomials)


def slow_table(ewaldcof: float, cutoff: float, pairlistdist: float):
    """The FP64 slow-term table of the precise pass (nbk_slow_table): (rows,
    step) where row k (SLOW_TABLE_ROW = 6 doubles) holds c0..c5 of
    phi_s(s) ~ sum c_n (s - k step)^n on s in [k step - step/2, k step + step/2];
    host-only."""
    L = dev_lib()
    rows = L.nbk_slow_table(ewaldcof, cutoff, pairlistdist, None, 0, None)
    if rows <= 0:
        raise NbkError(f"nbk_slow_table failed ({rows})")
    out = np.zeros((rows, SLOW_TABLE_ROW))
    step = C.c_double(0.0)
    rc = L.nbk_slow_table(ewaldcof, cutoff, pairlistdist, out.ctypes.data, rows, C.byref(step))
    if rc != rows:
        raise NbkError(f"nbk_slow_table failed ({rc})")
    return out, step.value


def measure_fp32_peak(device: int = 0) -> float:
    t = C.c_double(0)
    _dcheck(dev_lib().nbk_measure_fp32_peak(device, C.byref(t)), "nbk_measure_fp32_peak")
    return float(t.value)


def measure_fp64_peak(device: int = 0) -> float:
    t = C.c_double(0)
    _dcheck(dev_lib().nbk_measure_fp64_peak(device, C.byref(t)), "nbk_measure_fp64_peak")
    return float(t.value)


def pairs_from_tile_lists(tl, jatom, excl, storage):
    """Decodes exported tile lists into sorted uint64 keys i*storage + j."""
    keys = []
    lane = np.arange(32)
    for L in range(len(tl)):
        istart, js, je = tl[L, 0], tl[L, 1], tl[L, 2]
        if je < js:
            continue
        m = excl[js:je + 1]                                 # [nj, 32 lanes]
        t = np.arange(32)
        bits = (m[:, :, None] >> t[None, None, :]) & 1      # [nj, lane, t]
        jt, ln, tt = np.nonzero(bits)
        i = istart + ln
        j = jatom[js + jt] + ((ln + tt) & 31)
        keys.append(i.astype(np.uint64) * np.uint64(storage) + j.astype(np.uint64))
    if not keys:
        return np.zeros(0, dtype=np.uint64)
    k = np.concatenate(keys)
    k.sort()
    return k


# ---------------------------------------------------------------------------
# GPU-resident input marshaling
# ---------------------------------------------------------------------------
LOCAL_RECORD_WORDS = 32   # nbk_local_record (CudaLocalRecord) is 128 bytes


class ResidentLayout:
    """The per-atom arrays a GPU-resident integrator holds for one system, in
    buffer order (patch by patch, each patch's atoms in ascending global id or
    in the order `order_in_patch` gives), with the CudaLocalRecord of every
    patch -- built from a System and its Packed layout, on the host and as
    device tensors (`dev`). Patch assignment and slot ranges are the Packed
    layout's."""

    def __init__(self, system: System, packed: Packed, device=0, shuffle_seed=None):
        """device=None builds the host arrays only."""
        import torch
        a = system.arrays()
        n = system.natoms
        pa = packed.patches                       # numAtoms, numFreeAtoms, atomStart, id
        slot = packed.slotOfAtom
        start = pa[:, 2]
        patch_of = np.searchsorted(start, slot, side="right") - 1
        ids = np.lexsort((np.arange(n), patch_of))  # by patch, then by id
        if shuffle_seed is not None:
            rng = np.random.default_rng(shuffle_seed)
            off = 0
            for p in range(len(pa)):
                k = int(pa[p, 0])
                rng.shuffle(ids[off:off + k])
                off += k
        self.numPatches = len(pa)
        self.atomStorageSize = packed.atomStorageSize
        self.ids = ids.astype(np.int32)            # global id at each buffer position
        rec = np.zeros((len(pa), LOCAL_RECORD_WORDS), dtype=np.int32)
        counts = pa[:, 0]
        rec[:, 0] = np.arange(len(pa))
        rec[:, 1] = np.concatenate([[0], np.cumsum(counts)[:-1]])
        rec[:, 2] = start
        rec[:, 3] = counts
        rec[:, 4] = ((counts + 31) // 32) * 32
        self.records = rec
        pos = np.asarray(a["pos"], dtype=np.float64).reshape(-1, 3)
        self.pos = np.ascontiguousarray(pos[ids].T)              # [3, natoms]
        self.charge = np.asarray(a["charge"], dtype=np.float32)[ids]
        self.vdw = np.asarray(a["type"], dtype=np.int32)[ids]
        em = packed.exclIndexMaxDiff[slot]                      # (base, maxdiff) per atom id
        self.excl_by_atom = np.ascontiguousarray(em[:, ::-1], dtype=np.int32)
        # patch centres as fractional coordinates of an identity lattice
        # (so that the unscaled centre is exactly the Cartesian one)
        self.centres = np.ascontiguousarray(packed.patchCenter, dtype=np.float64)
        self.lattice = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], dtype=np.float64)
        self.qscale = float(np.sqrt(332.0636 * packed.coulomb_scaling))
        self.dev = None
        if device is None:
            return
        dev = torch.device("cuda", device)
        t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
        self.dev = {"records": t(rec), "x": t(self.pos[0]), "y": t(self.pos[1]),
                    "z": t(self.pos[2]), "charge": t(self.charge), "vdw": t(self.vdw),
                    "id": t(self.ids), "centres": t(self.centres)}

    def host_sort_order(self, packed: Packed):
        """The sort order that reproduces the Packed slot order exactly."""
        order = np.zeros(len(self.ids), dtype=np.int32)
        slot = packed.slotOfAtom[self.ids]
        for p in range(self.numPatches):
            b, k = self.records[p, 1], self.records[p, 3]
            if k == 0:
                continue
            local = slot[b:b + k] - self.records[p, 2]           # slot within patch
            order[b + local] = np.arange(k, dtype=np.int32)
        return order

    def sort_patch_atoms(self, sort_order, max_patch_atoms=None, status=None, stream=None):
        d = self.dev
        m = int(self.records[:, 3].max()) if max_patch_atoms is None else max_patch_atoms
        _dcheck(dev_lib().nbk_sort_patch_atoms(self.numPatches, _ptr(d["records"]), m,
                                               _ptr(d["x"]), _ptr(d["y"]), _ptr(d["z"]),
                                               _ptr(d["id"]), _ptr(sort_order), _ptr(status),
                                               stream), "nbk_sort_patch_atoms")

    def set_compute_positions(self, sort_order, xyzq, stream=None):
        d = self.dev
        lat = self.lattice.ctypes.data_as(C.POINTER(C.c_double))
        _dcheck(dev_lib().nbk_set_compute_positions(
            self.numPatches, _ptr(d["records"]), _ptr(d["centres"]), lat, _ptr(sort_order),
            self.qscale, _ptr(d["x"]), _ptr(d["y"]), _ptr(d["z"]), _ptr(d["charge"]),
            _ptr(xyzq), stream), "nbk_set_compute_positions")


# ---------------------------------------------------------------------------
# PME reciprocal space
# ---------------------------------------------------------------------------
def _lat(lattice, n):
    a = np.ascontiguousarray(np.asarray(lattice, dtype=np.float64).reshape(-1)[:n])
    assert a.size == n
    return a


class Pme:
    """PME reciprocal space on one GPU (nbk_pme_*): grid (K1, K2, K3), B-spline
    order 4, 6 or 8, Ewald coefficient ewaldcof. Atoms are device float4
    (fractional x, y, z in [0, 1), scaled charge); lattices are (a, b, c)."""

    def __init__(self, K, order, ewaldcof, device=0):
        g = PmeGrid(int(K[0]), int(K[1]), int(K[2]), int(order))
        h = C.c_void_p()
        _dcheck(dev_lib().nbk_pme_create(device, C.byref(g), float(ewaldcof), C.byref(h)),
                "nbk_pme_create")
        self._h = h
        self.K = tuple(int(k) for k in K)
        self.order = int(order)
        self.ewaldcof = float(ewaldcof)

    def close(self):
        if getattr(self, "_h", None) and _dev is not None:
            _dev.nbk_pme_destroy(self._h)
            self._h = None

    __del__ = close

    @staticmethod
    def atoms_from_positions(x, y, z, charge, qscale, lattice_abco, atoms, stream=None):
        """Device FP64 positions and FP32 charges -> fractional float4 atoms."""
        lat = _lat(lattice_abco, 12)
        n = int(x.numel()) if hasattr(x, "numel") else len(x)
        _dcheck(dev_lib().nbk_pme_atoms_from_positions(
            n, _ptr(x), _ptr(y), _ptr(z), _ptr(charge), float(qscale),
            lat.ctypes.data_as(C.POINTER(C.c_double)), _ptr(atoms), stream),
            "nbk_pme_atoms_from_positions")

    def spread(self, atoms, n, stream=None):
        _dcheck(dev_lib().nbk_pme_spread_charge(self._h, int(n), _ptr(atoms), stream),
                "nbk_pme_spread_charge")

    def solve(self, lattice, flags=NBK_ENERGY | NBK_VIRIAL, stream=None):
        lat = _lat(lattice, 9)
        _dcheck(dev_lib().nbk_pme_solve(self._h, lat.ctypes.data_as(C.POINTER(C.c_double)),
                                        flags, stream), "nbk_pme_solve")

    def gather(self, atoms, n, lattice, force, stream=None):
        lat = _lat(lattice, 9)
        _dcheck(dev_lib().nbk_pme_gather_force(self._h, int(n), _ptr(atoms),
                                               lat.ctypes.data_as(C.POINTER(C.c_double)),
                                               _ptr(force), stream), "nbk_pme_gather_force")

    def energy_virial(self, stream=None):
        e = C.c_double(0)
        v = (C.c_double * 9)()
        _dcheck(dev_lib().nbk_pme_get_energy_virial(self._h, C.byref(e), v, stream),
                "nbk_pme_get_energy_virial")
        return float(e.value), np.array(v[:], dtype=np.float64).reshape(3, 3)

    def self_energy(self, atoms, n, stream=None):
        e = C.c_double(0)
        _dcheck(dev_lib().nbk_pme_self_energy(self._h, int(n), _ptr(atoms), C.byref(e), stream),
                "nbk_pme_self_energy")
        return float(e.value)

    def compute(self, atoms, n, lattice, force, flags=NBK_ENERGY | NBK_VIRIAL, stream=None):
        """Spread, solve, gather: forces into `force` (device float3[n])."""
        self.spread(atoms, n, stream)
        self.solve(lattice, flags, stream)
        self.gather(atoms, n, lattice, force, stream)
