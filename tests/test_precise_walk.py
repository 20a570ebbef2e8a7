"""The precise kernel's walk over a tile's live words (host-only): a step-by-step
restatement of precisePass's enumeration in csrc/nbk_force.cu (the lanes'
inclusive counts, the binary search for the owner of a lane's first pair,
dropLowBits, walkNext), run over random and extreme tiles. Checks that every
interacting pair is taken exactly once, by the lane whose contiguous range of
the lane-major order holds it; that every lane index, shuffle source and bit
position stays in [0, 31]; and that a lane with no pair left (or none at all)
evaluates a real interacting pair, so that no distance given to the
reciprocal square root is 0."""
import numpy as np
import pytest

M32 = 0xFFFFFFFF


def popc(x):
    return bin(x & M32).count("1")


def ffs(x):
    """__ffs: 1-based position of the lowest set bit, 0 for 0."""
    x &= M32
    return 0 if x == 0 else (x & -x).bit_length()


def drop_low_bits(w, r):
    p = 0
    for step in (16, 8, 4, 2, 1):
        assert 0 <= p + step <= 31
        if popc(w & ((1 << (p + step)) - 1)) <= r:
            p += step
    return w & ((M32 << p) & M32)


def walk(live):
    """Runs the enumeration of one tile; returns the pairs (lane, step, i, t)
    taken by valid steps. live: 32 words, bit t of word i = pair (i, (i+t)&31)."""
    n = [popc(w) for w in live]
    incl = list(np.cumsum(n))
    excl = [incl[k] - n[k] for k in range(32)]
    total = int(incl[31])
    if total == 0:
        return []
    m = (total + 31) >> 5
    non_empty = sum(1 << k for k in range(32) if live[k])
    lanes = []
    for k in range(32):
        e0 = k * m
        cnt = min(m, max(0, total - e0))
        if e0 >= total:
            e0 = 0
        owner = 0
        for step in (16, 8, 4, 2, 1):
            src = owner + step - 1
            assert 0 <= src <= 31
            if incl[src] <= e0:
                owner += step
        assert 0 <= owner <= 31 and excl[owner] <= e0 < incl[owner]
        w = drop_low_bits(live[owner], e0 - excl[owner])
        assert w != 0
        lanes.append({"i": owner, "w": w, "cnt": cnt, "pi": owner, "pt": ffs(w) - 1})
    taken = []
    for s in range(m):
        for k, L in enumerate(lanes):
            valid = s < L["cnt"]
            if valid:
                assert L["w"] != 0
                L["pt"] = ffs(L["w"]) - 1
                L["pi"] = L["i"]
                L["w"] &= L["w"] - 1
            inext = ffs(non_empty & ((0xFFFFFFFE << L["i"]) & M32)) - 1
            assert -1 <= inext <= 31
            wn = live[inext & 31]
            if valid and L["w"] == 0 and inext >= 0:
                L["i"], L["w"] = inext, wn
            assert 0 <= L["pi"] <= 31 and 0 <= L["pt"] <= 31
            assert (live[L["pi"]] >> L["pt"]) & 1, "the evaluated pair is an interacting pair"
            if valid:
                taken.append((k, s, L["pi"], L["pt"]))
    return taken


def check(live):
    taken = walk(live)
    order = [(i, t) for i in range(32) for t in range(32) if (live[i] >> t) & 1]
    taken.sort(key=lambda v: (v[0], v[1]))
    assert [(i, t) for _, _, i, t in taken] == order


@pytest.mark.parametrize("seed", range(4))
def test_walk_takes_every_pair_once_in_range(seed):
    rng = np.random.default_rng(seed)
    for _ in range(500):
        dens = rng.choice([0.02, 0.1, 0.2, 0.4, 0.8, 1.0])
        bits = rng.random((32, 32)) < dens
        if rng.random() < 0.5:
            bits[rng.random(32) < 0.5] = False
        live = [int(sum(1 << t for t in range(32) if bits[i, t])) for i in range(32)]
        check(live)


def test_walk_extreme_tiles():
    check([M32] * 32)                 # 1,024 pairs: m = 32, every lane full
    check([1] + [0] * 31)             # one pair: 31 lanes repeat it with qq = 0
    check([0] * 31 + [1 << 31])       # the last lane's last bit
    check([0] * 31 + [M32])           # one owner for every lane's range
    check([M32 if k % 2 else 0 for k in range(32)])
    assert walk([0] * 32) == []
