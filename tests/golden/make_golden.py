"""Generates tests/golden/ref_pairmath.npz from the reference's own pair-math
functions (src/CudaComputeNonbondedInteractions.h), compiled host-side by
oracle/ref_pin/Makefile into oracle/_ref/libref_pairmath.so.

Run in a tree that has the reference sources:
    make -C oracle/ref_pin && python tests/golden/make_golden.py
The fixture is committed; the tests only read it.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CUTOFF, SWITCH, EWALD = 12.0, 10.0, 0.2579


def main():
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_pairmath.so"))
    rng = np.random.default_rng(20261203)
    n = 4000
    # distances from 1 A to just inside the cutoff, denser near the switch
    r = np.concatenate([rng.uniform(1.0, 12.0, n // 2), rng.uniform(9.5, 11.999, n // 4),
                        rng.uniform(1.0, 3.0, n - n // 2 - n // 4)])
    r2 = (r * r).astype(np.float32)
    qq = rng.uniform(-250.0, 250.0, n).astype(np.float32)
    sig = rng.uniform(2.0, 4.0, n)
    eps = rng.uniform(0.0, 0.2, n)
    B = (4.0 * eps * sig ** 6).astype(np.float32)
    A = (4.0 * eps * sig ** 12).astype(np.float32)
    # modified-pair LJ deltas (A14 - A, B14 - B) of mixed sign
    dA = (A * rng.uniform(-0.5, 0.5, n)).astype(np.float32)
    dB = (B * rng.uniform(-0.5, 0.5, n)).astype(np.float32)
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    out_nb = np.zeros((n, 5), dtype=np.float32)
    out_mod = np.zeros((n, 5), dtype=np.float32)
    for fn, a_, b_, out in ((lib.ref_nonbonded_pair, A, B, out_nb),
                            (lib.ref_modified_pair, dA, dB, out_mod)):
        fn.argtypes = [C.c_int] + [C.POINTER(C.c_float)] * 4 + [C.c_double] * 3 + [C.POINTER(C.c_float)]
        fn(n, fp(r2), fp(qq), fp(a_), fp(b_), CUTOFF, SWITCH, EWALD, fp(out))
    np.savez_compressed(os.path.join(HERE, "ref_pairmath.npz"), r2=r2, qq=qq, A=A, B=B, dA=dA,
                        dB=dB, out_nb=out_nb, out_mod=out_mod,
                        consts=np.array([CUTOFF, SWITCH, EWALD]))
    print("wrote", os.path.join(HERE, "ref_pairmath.npz"))


if __name__ == "__main__":
    main()
