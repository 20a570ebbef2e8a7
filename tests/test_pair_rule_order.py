"""The FP32 rounding order of the pair-set rule (host-only). The reference's
kernels form r^2 = dx*dx + dy*dy + dz*dz (src/CudaComputeNonbondedKernel.cu:
1225-1230) rounded as fma(dz, dz, fma(dx, dx, dy*dy)): on the mixed 20,000-atom
system sheared into a triclinic cell (tests/test_gpu_triclinic.py), their
refined lists hold the pair of slots (12435, 17456), whose r^2 is 182.249985
in that order and exactly plcutoff^2 = 182.25 in the order
fma(dz, dz, fma(dy, dy, dx*dx)) (observed on a B200 through the reference
harness; the GPU test compares the whole pair sets). The oracle, which the GPU
path is tested against bit for bit, must list it too."""
import importlib.util
import os

import numpy as np

import nbk
import oracle
from helpers import PARAMS, mixed_box, unordered_keys

HERE = os.path.dirname(os.path.abspath(__file__))
PAIR = (12435, 17456)


def _triclinic():
    spec = importlib.util.spec_from_file_location(
        "triclinic_cell", os.path.join(HERE, "test_gpu_triclinic.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    p = nbk.Packed(mixed_box(natoms=20000))
    return mod.sheared(p, mod.SHEAR)


def _fma32(a, b, c):
    """FP32 fma from exact float64 arithmetic: a*b is exact in float64 and, for
    these magnitudes, so is the sum, which is then rounded once to FP32."""
    return np.float32(np.float64(a) * np.float64(b) + np.float64(c))


def test_boundary_pair_follows_the_reference_order():
    t = _triclinic()
    n = t.atomStorageSize
    keys, _ = oracle.Oracle(t, PARAMS).pairs()
    listed = unordered_keys(keys, n)
    key = np.uint64(PAIR[0]) * np.uint64(n) + np.uint64(PAIR[1])
    assert key in set(listed.tolist())
    # the pair's FP32 geometry in compute order (i in the compute's first patch)
    i, j = PAIR
    start = t.patches[:, 2]
    end = start + (t.patches[:, 0] + 31) // 32 * 32      # slots of each patch, padded to 32

    def patch_of(slot):
        return int(np.flatnonzero((start <= slot) & (slot < end))[0])

    c = next(k for k in range(t.numComputes)
             if tuple(t.computes_patch[k]) == (patch_of(i), patch_of(j)))
    o = t.computes_offset[c].astype(np.float32)
    L = t.lattice.astype(np.float32)
    sh = [_fma32(o[2], L[2, d], _fma32(o[0], L[0, d], np.float32(o[1] * L[1, d]))) for d in range(3)]
    d = [np.float32(t.xyzq[j, k] - np.float32(t.xyzq[i, k] + sh[k])) for k in range(3)]
    pl2 = np.float32(PARAMS.pairlistdist) * np.float32(PARAMS.pairlistdist)
    r2_ref = _fma32(d[2], d[2], _fma32(d[0], d[0], np.float32(d[1] * d[1])))
    r2_other = _fma32(d[2], d[2], _fma32(d[1], d[1], np.float32(d[0] * d[0])))
    assert r2_ref < pl2 and not (r2_other < pl2), (float(r2_ref), float(r2_other))
