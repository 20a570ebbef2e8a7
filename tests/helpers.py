"""Shared helpers of the test suite: system set-up, GPU runs and error norms."""
import numpy as np

import nbk
import oracle

PARAMS = nbk.NonbondedParams()
ALL = nbk.NBK_ENERGY | nbk.NBK_VIRIAL | nbk.NBK_SLOW

# tolerances (relative to the FP64 oracle)
FORCE_RMS_TOL = 1e-5      # RMS relative force error
ENERGY_TOL = 1e-6         # relative error of each energy term
VIRIAL_TOL = 1e-6         # Frobenius-relative virial error


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


# ---------------------------------------------------------------------------
# packed-system variants for the pairlist refinement's edge cases
# ---------------------------------------------------------------------------
class PackedVariant:
    """A Packed system with some of its arrays replaced: the attributes the
    oracle and the reference harness read and the view the device library
    reads both point at the replacements. Only for test inputs."""

    _FIELDS = {"atomIndex": "atomIndex", "exclIndexMaxDiff": "exclIndexMaxDiff",
               "exclusionBits": "exclusionBits", "patches": "patches", "xyzq": "xyzq"}
    _DTYPES = {"exclusionBits": np.uint32, "xyzq": np.float32}

    def __init__(self, packed, **arrays):
        self.__dict__.update(packed.__dict__)
        self._base = packed            # keeps the host-side storage alive
        self._keep = []
        v = nbk.PackedView.from_buffer_copy(packed.v)
        for name, arr in arrays.items():
            arr = np.ascontiguousarray(arr, dtype=self._DTYPES.get(name, np.int32))
            self._keep.append(arr)
            setattr(self, name, arr)
            field = self._FIELDS[name]
            setattr(v, field, arr.ctypes.data_as(type(getattr(v, field))))
            if name == "exclusionBits":
                v.numExclusionWords = len(arr)
        self.v = v


def exclusion_lists(system):
    """Per atom: the sorted offsets {0} U {partner - atom} of its full exclusions."""
    partners = [[0] for _ in range(system.natoms)]
    for x, y in system.arrays()["fullExcl"]:
        partners[x].append(int(y) - int(x))
        partners[y].append(int(x) - int(y))
    return partners


def renumbered(packed, perm):
    """The packed system with global atom index g renamed perm[g]: atomIndex
    and the (base, maxdiff) exclusion bit array re-encoded for the new
    numbering, so that exactly the same pairs stay excluded."""
    offs = exclusion_lists(packed.system)
    lists, base, maxdiff, total = {}, [], [], 0
    atom_list = np.empty(len(offs), dtype=np.int64)
    for a, lst in enumerate(offs):
        key = tuple(sorted({int(perm[a + d]) - int(perm[a]) for d in lst}))
        k = lists.get(key)
        if k is None:
            k = lists[key] = len(base)
            md = max(-key[0], key[-1])
            base.append(total + md)
            maxdiff.append(md)
            total += 2 * md + 1
        atom_list[a] = k
    bits = np.zeros((total + 31) // 32, dtype=np.uint32)
    for key, k in lists.items():
        for d in key:
            b = base[k] + d
            bits[b >> 5] |= np.uint32(1 << (b & 31))
    old = packed.atomIndex.astype(np.int64)
    em = np.stack([np.asarray(base, np.int64)[atom_list[old]],
                   np.asarray(maxdiff, np.int64)[atom_list[old]]], axis=1)
    return PackedVariant(packed, atomIndex=np.asarray(perm, np.int64)[old], exclIndexMaxDiff=em,
                         exclusionBits=bits)


def molecule_boundaries(system):
    """Global indices b such that no full exclusion joins an atom below b to
    one at or above b."""
    cross = np.zeros(system.natoms + 1, dtype=np.int64)
    for x, y in system.arrays()["fullExcl"]:
        lo, hi = min(x, y), max(x, y)
        cross[lo + 1] += 1
        cross[hi + 1] -= 1
    return np.flatnonzero(np.cumsum(cross) == 0)


def unordered_keys(keys, storage):
    """Pair keys i*storage + j as sorted keys of unordered pairs (min, max)."""
    n = np.uint64(storage)
    i, j = keys // n, keys % n
    return np.sort(np.minimum(i, j) * n + np.maximum(i, j))


def reference_pairs(ref, xyzq, storage):
    """A pairlist evaluation through the reference kernels (a refgpu.RefGpu
    after setup): the unordered pairs of their refined tile lists and the
    reference's excluded-pair count."""
    ref.eval(1, 1, 1, 1, xyzq)
    tl, ja, ex, nexcl = ref.tile_lists()
    return unordered_keys(nbk.pairs_from_tile_lists(tl, ja, ex, storage), storage), nexcl
