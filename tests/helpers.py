"""Shared helpers of the test suite: system set-up, GPU runs and error norms."""
import numpy as np

import nbk
import oracle

PARAMS = nbk.NonbondedParams()
ALL = nbk.NBK_ENERGY | nbk.NBK_VIRIAL | nbk.NBK_SLOW

# tolerances (relative to the FP64 oracle)
FORCE_RMS_TOL = 1e-5      # RMS relative force error
ENERGY_TOL = 1e-6         # relative error of each energy term (FP64 energy mode; LJ always)
VIRIAL_TOL = 1e-6         # Frobenius-relative virial error
# FP32 energy mode: each electrostatic pair energy carries ~1e-7 relative FP32
# error, so a total that cancels to 1/2e4 of the sum of |pair energies| (the
# random-orientation water here) is resolved to ~1e-5 of itself.
FP32_ELEC_ENERGY_TOL = 5e-5
# FP32 energy mode: the virial is sum F_i (x) x_i over FP32 pair forces. Near
# the cutoff the electrostatic split rc^-3 - r^-3 cancels, which leaves the
# slow virial (small next to its terms) at about 1e-6 of itself; the FP64
# energy/virial mode (NBK_ENERGY_FP64) holds VIRIAL_TOL with a wide margin.
FP32_VIRIAL_TOL = 2e-6


def water_box(seed=1, nwater=3000, box=44.8):
    return nbk.System(nbk.NBK_SYS_WATER, seed, 3 * nwater, 0.0, box=(box, box, box))


def mixed_box(seed=2, natoms=20000, frac=0.3, box=None):
    return nbk.System(nbk.NBK_SYS_MIXED, seed, natoms, frac, box=box)


def rms_rel(a, b):
    num = np.sqrt(((a - b) ** 2).sum())
    den = np.sqrt((b ** 2).sum())
    return num / den if den > 0 else num


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


class GpuRun:
    """Runs the GPU path on a packed system and returns host results."""

    def __init__(self, packed, params=PARAMS, device=0):
        import torch
        self.torch = torch
        self.packed = packed
        self.params = params
        self.lj = packed.system.lj_table()
        self.nb = nbk.Nonbonded(params, self.lj, device)
        self.nb.setup(packed)
        n = packed.atomStorageSize
        self.dF = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        self.dS = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        self.dX = torch.zeros((6, n), dtype=torch.int64, device="cuda")

    def build(self):
        self.nb.build_tile_lists(self.packed)

    def eval(self, flags, xyzq=None):
        xyzq = self.packed.xyzq if xyzq is None else xyzq
        self.nb.force(self.packed, flags, xyzq=xyzq, d_forces=self.dF, d_forcesSlow=self.dS,
                      d_fixed=self.dX)
        ve = self.nb.virial_energy(flags)
        self.torch.cuda.synchronize()
        F = self.dX[:3].T.cpu().numpy().astype(np.float64) / nbk.FORCE_FIXED_SCALE
        S = self.dX[3:].T.cpu().numpy().astype(np.float64) / nbk.FORCE_FIXED_SCALE
        res = dict(energyVdw=ve.energyVdw, energyElec=ve.energyElec, energySlow=ve.energySlow,
                   virial=np.array(ve.virial).reshape(3, 3),
                   virialSlow=np.array(ve.virialSlow).reshape(3, 3))
        return F, S, res, self.dX.cpu().numpy().copy()


def compare(F, S, res, Fo, So, ro, real):
    """Error table of a GPU result against the oracle on the real atom slots."""
    out = dict(force=rms_rel(F[real], Fo[real]), slow=rms_rel(S[real], So[real]))
    for k in ("energyVdw", "energyElec", "energySlow"):
        out[k] = rel(res[k], ro[k])
    out["virial"] = rms_rel(res["virial"], ro["virial"])
    out["virialSlow"] = rms_rel(res["virialSlow"], ro["virialSlow"])
    return out


def real_slots(packed):
    mask = np.zeros(packed.atomStorageSize, dtype=bool)
    mask[packed.slotOfAtom] = True
    return mask
