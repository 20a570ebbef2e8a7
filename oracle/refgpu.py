"""ctypes wrapper of oracle/_ref/libref_nbgpu.so: the reference's own CUDA
tile-list and nonbonded kernels (src/CudaTileListKernel.cu,
src/CudaComputeNonbondedKernel.cu) built from the reference tree by
oracle/ref_gpu/Makefile, driven in the order CudaComputeNonbonded::launchWork
uses (src/CudaComputeNonbonded.C:1440-1530), and its PME kernels
(src/CudaPmeSolverUtilKernel.cu) driven as CudaPmeOneDevice does
(src/CudaPmeSolverUtil.C:1364-1650).

Test infrastructure: the tests use it to pin the product's tile-list pair sets
and forces against the reference kernels themselves and to time the
reference's plain GPU path on the same device. The product never imports it.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref_nbgpu.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        vp, ip, dp, fp = C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_float)
        L.refgpu_last_error.restype = C.c_char_p
        L.refgpu_create.argtypes = [ip, dp, ip, dp, dp, ip, C.POINTER(vp)]
        L.refgpu_setup.argtypes = [vp, ip, vp, ip, vp, ip, ip, vp, vp, vp, ip, vp]
        L.refgpu_eval.argtypes = [vp, ip, ip, ip, ip, fp, vp]
        L.refgpu_sync.argtypes = [vp]
        L.refgpu_stream.argtypes = [vp]
        L.refgpu_stream.restype = vp
        L.refgpu_set_stream.argtypes = [vp, vp]
        L.refgpu_device_xyzq.argtypes = [vp]
        L.refgpu_device_xyzq.restype = vp
        L.refgpu_results.argtypes = [vp, vp, vp, vp]
        L.refgpu_tile_list_sizes.argtypes = [vp, C.POINTER(C.c_int)]
        L.refgpu_tile_lists.argtypes = [vp, vp, vp, vp]
        L.refgpu_destroy.argtypes = [vp]
        L.refpme_last_error.restype = C.c_char_p
        L.refpme_create.argtypes = [ip, ip, ip, ip, C.c_double, fp, fp, fp, C.POINTER(vp)]
        L.refpme_compute.argtypes = [vp, vp, ip, dp, C.c_double, ip, vp, vp]
        L.refpme_energy_virial.argtypes = [vp, dp]
        L.refpme_destroy.argtypes = [vp]
        _lib = L
    return _lib


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: {lib().refgpu_last_error().decode()}")


class RefGpu:
    """One reference CudaTileListKernel + CudaComputeNonbondedKernel pair on
    its own stream. do_table=1 is the reference's texture-table mode (its
    choice whenever slow forces are on); 0 is direct math."""

    def __init__(self, params, lj, do_table=1, device=0):
        dim, A, B = lj[0], np.ascontiguousarray(lj[1], np.float64), np.ascontiguousarray(lj[2], np.float64)
        prm = np.array([params.cutoff, params.switchdist, params.pairlistdist, params.ewaldcof,
                        params.scaling, params.slowScale], dtype=np.float64)
        h = C.c_void_p()
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        _check(lib().refgpu_create(device, dp(prm), dim, dp(A), dp(B), do_table, C.byref(h)),
               "refgpu_create")
        self._h = h
        self._keep = (A, B, prm)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.refgpu_destroy(self._h)
            self._h = None

    @property
    def stream_ptr(self) -> int:
        return lib().refgpu_stream(self._h) or 0

    def set_stream(self, stream_ptr):
        """Evaluate on a caller's CUDA stream (an int handle; 0: own stream)."""
        _check(lib().refgpu_set_stream(self._h, stream_ptr or None), "refgpu_set_stream")

    def setup(self, packed):
        self.n = packed.atomStorageSize
        self._arrs = [np.ascontiguousarray(packed.patches, np.int32),
                      np.ascontiguousarray(packed.computes, np.int32),
                      np.ascontiguousarray(packed.vdwTypes, np.int32),
                      np.ascontiguousarray(packed.exclIndexMaxDiff, np.int32),
                      np.ascontiguousarray(packed.atomIndex, np.int32),
                      np.ascontiguousarray(packed.exclusionBits, np.uint32)]
        pa, co, vt, em, ai, eb = self._arrs
        _check(lib().refgpu_setup(self._h, packed.numPatches, pa.ctypes.data, packed.numComputes,
                                  co.ctypes.data, self.n, packed.maxTileListLen, vt.ctypes.data,
                                  em.ctypes.data, ai.ctypes.data, len(eb), eb.ctypes.data),
               "refgpu_setup")
        self.lattice = np.ascontiguousarray(packed.lattice, np.float32).reshape(9)

    def eval(self, pairlist, energy, virial, slow, xyzq=None, lattice=None):
        """xyzq: host float32 [n,4] array, or None for the positions already
        on the device (the kernels alone; not allowed on a pairlist step)."""
        lat = self.lattice if lattice is None else np.ascontiguousarray(lattice, np.float32).reshape(9)
        ptr = None
        if xyzq is not None:
            assert xyzq.dtype == np.float32 and xyzq.flags.c_contiguous and xyzq.size == 4 * self.n
            ptr = xyzq.ctypes.data
        _check(lib().refgpu_eval(self._h, int(pairlist), int(energy), int(virial), int(slow),
                                 lat.ctypes.data_as(C.POINTER(C.c_float)), ptr), "refgpu_eval")

    def sync(self):
        _check(lib().refgpu_sync(self._h), "refgpu_sync")

    def results(self):
        F = np.zeros((self.n, 4), np.float32)
        S = np.zeros((self.n, 4), np.float32)
        ve = np.zeros(21, np.float64)
        _check(lib().refgpu_results(self._h, F.ctypes.data, S.ctypes.data, ve.ctypes.data),
               "refgpu_results")
        return F, S, ve

    def tile_lists(self):
        sz = (C.c_int * 3)()
        _check(lib().refgpu_tile_list_sizes(self._h, sz), "refgpu_tile_list_sizes")
        nl, nj, nexcl = sz[0], sz[1], sz[2]
        tl = np.zeros((max(nl, 1), 12), np.int32)
        ja = np.zeros(max(nj, 1), np.int32)
        ex = np.zeros((max(nj, 1), 32), np.uint32)
        _check(lib().refgpu_tile_lists(self._h, tl.ctypes.data, ja.ctypes.data, ex.ctypes.data),
               "refgpu_tile_lists")
        return tl[:nl], ja[:nj], ex[:nj], nexcl


def _pcheck(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what}: {lib().refpme_last_error().decode()}")


class RefPme:
    """The reference's single-device PME kernels on one grid: K (K1, K2, K3),
    B-spline order, Ewald coefficient and the B-spline moduli per dimension
    (the values of the reference's compute_b_moduli, passed in FP32 as it
    does)."""

    def __init__(self, K, order, kappa, moduli):
        bm = [np.ascontiguousarray(m, np.float32) for m in moduli]
        self._keep = bm
        h = C.c_void_p()
        fpp = C.POINTER(C.c_float)
        _pcheck(lib().refpme_create(int(K[0]), int(K[1]), int(K[2]), int(order), float(kappa),
                                    bm[0].ctypes.data_as(fpp), bm[1].ctypes.data_as(fpp),
                                    bm[2].ctypes.data_as(fpp), C.byref(h)), "refpme_create")
        self._h = h

    def __del__(self):
        _l = _lib
        if getattr(self, "_h", None) and _l is not None:
            _l.refpme_destroy(self._h)
            self._h = None

    def compute(self, atoms_ptr, n, lattice, forces_ptr, energy_virial=True, stream=None):
        """atoms_ptr: device float4[n] fractional atoms; lattice: 3x3 rows a,
        b, c; forces_ptr: device float3[n] (fractional-gradient forces)."""
        L = np.asarray(lattice, np.float64).reshape(3, 3)
        recip = np.ascontiguousarray(np.linalg.inv(L).T)      # rows a*, b*, c*
        vol = abs(float(np.linalg.det(L)))
        _pcheck(lib().refpme_compute(self._h, atoms_ptr, int(n),
                                     recip.reshape(-1).ctypes.data_as(C.POINTER(C.c_double)), vol,
                                     int(energy_virial), forces_ptr, stream), "refpme_compute")

    def energy_virial(self):
        out = np.zeros(7, np.float64)
        _pcheck(lib().refpme_energy_virial(self._h, out.ctypes.data_as(C.POINTER(C.c_double))),
                "refpme_energy_virial")
        return out
