"""Python face of the FP64 oracle (oracle/nbk_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker. The product path never imports
this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
NOUT = 25


class OracleSystem(C.Structure):
    _fields_ = [("atomStorageSize", C.c_int), ("numPatches", C.c_int), ("numComputes", C.c_int),
                ("vdwDim", C.c_int),
                ("xyzq", C.c_void_p), ("patches", C.c_void_p), ("computePatch", C.c_void_p),
                ("computeOffset", C.c_void_p), ("lattice", C.c_void_p), ("vdwTypes", C.c_void_p),
                ("atomIndex", C.c_void_p), ("exclIndexMaxDiff", C.c_void_p),
                ("exclBits", C.c_void_p), ("numExclWords", C.c_longlong),
                ("ljA", C.c_void_p), ("ljB", C.c_void_p), ("ljA14", C.c_void_p),
                ("ljB14", C.c_void_p),
                ("cutoff", C.c_double), ("switchdist", C.c_double), ("ewaldcof", C.c_double),
                ("scaling", C.c_double), ("scale14", C.c_double),
                ("cutoff2f", C.c_float), ("plcutoff2f", C.c_float)]


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(_HERE, "libnbk_oracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/libnbk_oracle.so is not built (make -C oracle)")
        L = C.CDLL(path)
        L.oracle_pairs.restype = C.c_longlong
        L.oracle_pairs.argtypes = [C.POINTER(OracleSystem), C.c_void_p, C.POINTER(C.c_longlong)]
        L.oracle_nonbonded.argtypes = [C.POINTER(OracleSystem), C.c_int, C.c_int, C.c_void_p,
                                       C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_nonbonded_sub.argtypes = [C.POINTER(OracleSystem), C.c_int, C.c_int, C.c_int,
                                           C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_num_threads.restype = C.c_int
        L.oracle_adjoint.restype = C.c_double
        L.oracle_adjoint.argtypes = [C.POINTER(OracleSystem), C.c_void_p, C.c_void_p, C.c_double,
                                     C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p]
        L.oracle_loss_local.restype = C.c_double
        L.oracle_loss_local.argtypes = [C.POINTER(OracleSystem), C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_double, C.c_double, C.c_double]
        L.oracle_near_cutoff.restype = C.c_int
        L.oracle_near_cutoff.argtypes = [C.POINTER(OracleSystem), C.c_int, C.c_float]
        _lib = L
    return _lib


class Oracle:
    """Holds contiguous copies of one packed system's inputs for the oracle."""

    def __init__(self, packed, params, lj=None):
        """packed: nbk.Packed; params: nbk.NonbondedParams; lj: (dim, A, B, A14, B14)."""
        self.packed = packed
        self.params = params
        if lj is None:
            lj = packed.system.lj_table()
        dim, A, B, A14, B14 = lj
        self._keep = []

        def keep(a, dtype):
            a = np.ascontiguousarray(a, dtype=dtype)
            self._keep.append(a)
            return a.ctypes.data

        s = OracleSystem()
        s.atomStorageSize = packed.atomStorageSize
        s.numPatches = packed.numPatches
        s.numComputes = packed.numComputes
        s.vdwDim = dim
        s.xyzq = keep(np.array(packed.xyzq, dtype=np.float32, copy=True), np.float32)
        s.patches = keep(packed.patches, np.int32)
        s.computePatch = keep(packed.computes_patch, np.int32)
        s.computeOffset = keep(packed.computes_offset, np.float32)
        s.lattice = keep(packed.lattice.reshape(-1), np.float32)
        s.vdwTypes = keep(packed.vdwTypes, np.int32)
        s.atomIndex = keep(packed.atomIndex, np.int32)
        s.exclIndexMaxDiff = keep(packed.exclIndexMaxDiff, np.int32)
        s.exclBits = keep(packed.exclusionBits, np.uint32)
        s.numExclWords = len(packed.exclusionBits)
        s.ljA, s.ljB = keep(A, np.float64), keep(B, np.float64)
        s.ljA14, s.ljB14 = keep(A14, np.float64), keep(B14, np.float64)
        s.cutoff, s.switchdist = params.cutoff, params.switchdist
        s.ewaldcof, s.scaling, s.scale14 = params.ewaldcof, params.scaling, params.scale14
        s.cutoff2f = np.float32(params.cutoff) * np.float32(params.cutoff)
        s.plcutoff2f = np.float32(params.pairlistdist) * np.float32(params.pairlistdist)
        self.s = s
        self.mod = np.ascontiguousarray(packed.modified)
        self.exc = np.ascontiguousarray(packed.excluded)

    def pairs(self):
        """Sorted uint64 keys i_slot*storage + j_slot of the listed pairs, and
        the number of excluded pairs within the pairlist cutoff."""
        L = lib()
        nex = C.c_longlong(0)
        n = L.oracle_pairs(C.byref(self.s), None, C.byref(nex))
        keys = np.empty(n, dtype=np.uint64)
        L.oracle_pairs(C.byref(self.s), keys.ctypes.data, None)
        keys.sort()
        return keys, int(nex.value)

    def forces(self, mode=1):
        """mode 1: nonbonded kernel semantics; 2: corrections only; 3: both.
        Returns (F[storage,3], Fslow[storage,3], dict of energies/virials)."""
        L = lib()
        n = self.packed.atomStorageSize
        F = np.zeros((n, 3))
        Fs = np.zeros((n, 3))
        out = np.zeros(NOUT)
        rc = L.oracle_nonbonded(C.byref(self.s), mode, len(self.mod), self.mod.ctypes.data,
                                len(self.exc), self.exc.ctypes.data, F.ctypes.data,
                                Fs.ctypes.data, out.ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle_nonbonded failed")
        res = dict(energyVdw=out[0], energyElec=out[1], energySlow=out[2],
                   virial=out[3:12].reshape(3, 3).copy(), virialSlow=out[12:21].reshape(3, 3).copy(),
                   pairs=int(out[21]),
                   absVdw=out[22], absElec=out[23], absSlow=out[24])
        return F, Fs, res

    def eval_range(self, c0=0, c1=-1):
        """Evaluates computes [c0, c1) on all threads (energies, virial, forces in
        FP64) and returns the number of pairs within the cutoff: the CPU
        baseline's unit of work."""
        n = self.packed.atomStorageSize
        if not hasattr(self, "_bufF"):
            self._bufF = np.zeros((n, 3))
            self._bufS = np.zeros((n, 3))
            self._out = np.zeros(NOUT)
        rc = lib().oracle_nonbonded_sub(C.byref(self.s), 1, c0, c1, 0, None, 0, None,
                                        self._bufF.ctypes.data, self._bufS.ctypes.data,
                                        self._out.ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle_nonbonded_sub failed")
        return int(self._out[21])


    # ---- adjoint -----------------------------------------------------------
    def adjoint(self, wF, wS, cV, cE, cS, grads=True):
        """FP64 loss L = sum wF.F_fast + sum wS.F_slow + cV E_vdw + cE E_elec +
        cS E_slow over the nonbonded pairs, and its gradient: (L, gX[n,3],
        gQ[n] w.r.t. the scaled charges, gA[dim,dim], gB[dim,dim] w.r.t. the
        scaled LJ table entries at ordered type pairs)."""
        n = self.packed.atomStorageSize
        dim = self.s.vdwDim
        wF = np.ascontiguousarray(wF, dtype=np.float64)
        wS = np.ascontiguousarray(wS, dtype=np.float64)
        out = [np.zeros((n, 3)), np.zeros(n), np.zeros((dim, dim)), np.zeros((dim, dim))]
        ptr = [o.ctypes.data if grads else None for o in out]
        L = lib().oracle_adjoint(C.byref(self.s), wF.ctypes.data, wS.ctypes.data, cV, cE, cS, *ptr)
        return (L, *out) if grads else L

    def loss_local(self, slot, wF, wS, cV, cE, cS):
        wF = np.ascontiguousarray(wF, dtype=np.float64)
        wS = np.ascontiguousarray(wS, dtype=np.float64)
        return lib().oracle_loss_local(C.byref(self.s), int(slot), wF.ctypes.data, wS.ctypes.data,
                                       cV, cE, cS)

    def near_cutoff(self, slot, tol):
        return lib().oracle_near_cutoff(C.byref(self.s), int(slot), float(tol))

    @property
    def xyzq(self):
        """The oracle's own (writable) copy of the positions and charges."""
        return self._keep[0]


def num_threads() -> int:
    return int(lib().oracle_num_threads())
