"""FP64 restatement of NAMD's smooth particle-mesh Ewald reciprocal space, and a
direct Ewald reciprocal sum that pins it.

Test infrastructure only: the tests, smoke() and bench.py's CPU leg use it as
the checker; the product (libnbk.so, nbk_pme_*) never calls it.

Restated from the reference:
  - fractional atoms: ComputePmeCUDA::sendAtoms, src/ComputePmeCUDA.C:281-300
    (w = (r - origin) . a_r, shifted into [0, 1) by w - (floor(w + 1/2) - 1/2),
    rounded to FP32);
  - grid cell and weights: spread_charge_kernel / gather_force,
    src/CudaPmeSolverUtilKernel.cu:440-470,725-760 (f = K * w in FP32, cell =
    (int) f, fraction f - cell) and calc_one_theta / calc_theta_dtheta,
    src/CudaPmeSolverUtilKernel.cu:329-424 (order-n B-spline weights on points
    cell + k, k = 0..n-1, by the recursion raising the order one step at a
    time; derivatives from the order n-1 weights);
  - B-spline moduli: compute_b_moduli / dftmod, src/PmeKSpace.C:22-61;
  - influence function, energy and virial: scalar_sum_kernel,
    src/CudaPmeSolverUtilKernel.cu:74-325 (half-complex grid, weight 1/2 on the
    k1 = 0 and k1 = K1/2 planes, energy = sum / 2, virial = -sum / 2 of
    fac (2 (pi^2/beta^2 + 1/m^2) m_a m_b - delta_ab));
  - force: -q (f1 K1 a_r + f2 K2 b_r + f3 K3 c_r), gather_force + the
    conversion of src/ComputePmeCUDA.C:640-652;
  - self energy: -beta/sqrt(pi) sum q^2, src/CudaPmeSolverUtilKernel.cu:1192-1216.
The direct sum is the textbook Ewald reciprocal energy
(1/(2 pi V)) sum_{m != 0} exp(-pi^2 m^2 / beta^2) / m^2 |S(m)|^2 and its
forces, which smooth PME approximates.
"""
import numpy as np


def reciprocal(lattice):
    """Rows a_r, b_r, c_r of the reciprocal lattice of rows a, b, c; volume."""
    L = np.asarray(lattice, dtype=np.float64).reshape(3, 3)
    a, b, c = L
    vol = float(np.dot(a, np.cross(b, c)))
    return np.array([np.cross(b, c), np.cross(c, a), np.cross(a, b)]) / vol, vol


def fractional_atoms(pos, charge, lattice, origin=(0.0, 0.0, 0.0), qscale=1.0):
    """float32 [n, 4] atoms as ComputePmeCUDA sends them."""
    R, _ = reciprocal(lattice)
    p = np.asarray(pos, dtype=np.float64) - np.asarray(origin, dtype=np.float64)
    w = p @ R.T
    w = w - (np.floor(w + 0.5) - 0.5)
    out = np.zeros((len(p), 4), dtype=np.float32)
    out[:, :3] = w.astype(np.float32)
    out[:, :3] -= (out[:, :3] >= np.float32(1.0)).astype(np.float32)
    out[:, 3] = (np.asarray(charge, dtype=np.float32).astype(np.float64) * qscale).astype(np.float32)
    return out


def theta(w, order):
    """B-spline weights [n, order] on the points cell + k (FP64)."""
    w = np.asarray(w, dtype=np.float64)
    t = np.zeros(w.shape + (order,))
    t[..., 1] = w
    t[..., 0] = 1.0 - w
    for k in range(3, order + 1):
        div = 1.0 / (k - 1)
        t[..., k - 1] = div * w * t[..., k - 2]
        for j in range(1, k - 1):
            t[..., k - j - 1] = div * ((w + j) * t[..., k - j - 2] + (k - j - w) * t[..., k - j - 1])
        t[..., 0] = div * (1.0 - w) * t[..., 0]
    return t


def dtheta(w, order):
    t1 = theta(w, order - 1)
    d = np.zeros(np.shape(w) + (order,))
    d[..., 0] = -t1[..., 0]
    for j in range(1, order - 1):
        d[..., j] = t1[..., j - 1] - t1[..., j]
    d[..., order - 1] = t1[..., order - 2]
    return d


def b_moduli(K, order):
    """1 / |DFT of the B-spline weights at w = 0|^2 (compute_b_moduli)."""
    th = theta(np.array([0.0]), order)[0]
    k = np.arange(K)[:, None]
    j = np.arange(order)[None, :]
    arg = 2.0 * np.pi * k * j / K
    s1 = (th[None, :] * np.cos(arg)).sum(1)
    s2 = (th[None, :] * np.sin(arg)).sum(1)
    return 1.0 / (s1 * s1 + s2 * s2)


def grid_cells(atoms, K):
    """Cell indices and fractions per dimension, in FP32 as the device forms them."""
    cells, fracs = [], []
    for d in range(3):
        f = np.float32(K[d]) * atoms[:, d].astype(np.float32)
        c = f.astype(np.int64)                    # truncation, f >= 0
        cells.append(c)
        fracs.append((f - c.astype(np.float32)).astype(np.float64))
    return cells, fracs


def pme(atoms, lattice, K, order, beta):
    """Smooth PME reciprocal energy, virial (3x3, sum r (x) F) and forces [n, 3]."""
    atoms = np.asarray(atoms, dtype=np.float32)
    K1, K2, K3 = (int(k) for k in K)
    R, vol = reciprocal(lattice)
    (cx, cy, cz), (wx, wy, wz) = grid_cells(atoms, K)
    q = atoms[:, 3].astype(np.float64)
    tx, ty, tz = theta(wx, order), theta(wy, order), theta(wz, order)
    Q = np.zeros((K3, K2, K1))
    o = np.arange(order)
    ix = (cx[:, None] + o[None, :]) % K1
    iy = (cy[:, None] + o[None, :]) % K2
    iz = (cz[:, None] + o[None, :]) % K3
    for c in range(order):
        for b in range(order):
            v = q[:, None] * tx * ty[:, b:b + 1] * tz[:, c:c + 1]
            np.add.at(Q, (iz[:, c:c + 1].repeat(order, 1), iy[:, b:b + 1].repeat(order, 1), ix), v)
    S = np.fft.rfftn(Q)                           # (K3, K2, K1/2+1), x fastest
    nh = K1 // 2 + 1
    k1 = np.arange(nh)[None, None, :]
    k2 = np.arange(K2)[None, :, None]
    k3 = np.arange(K3)[:, None, None]
    k2s = np.where(k2 <= K2 // 2, k2, k2 - K2)
    k3s = np.where(k3 <= K3 // 2, k3, k3 - K3)
    m = [R[0, d] * k1 + R[1, d] * k2s + R[2, d] * k3s for d in range(3)]
    msq = m[0] ** 2 + m[1] ** 2 + m[2] ** 2
    msq[0, 0, 0] = 1.0
    bm1, bm2, bm3 = b_moduli(K1, order), b_moduli(K2, order), b_moduli(K3, order)
    th3 = bm1[np.arange(nh)][None, None, :] * bm2[None, :, None] * bm3[:, None, None]
    piEwald = (np.pi / beta) ** 2
    C = np.exp(-piEwald * msq) / (np.pi * vol) / msq
    C[0, 0, 0] = 0.0
    wgt = np.full(nh, 2.0)
    wgt[0] = 1.0
    if K1 % 2 == 0:
        wgt[K1 // 2] = 1.0
    fac = wgt[None, None, :] * np.abs(S) ** 2 * th3 * C
    energy = 0.5 * fac.sum()
    vir = 2.0 * (piEwald + 1.0 / msq)
    W = np.zeros((3, 3))
    for a in range(3):
        for b in range(3):
            W[a, b] = -0.5 * (fac * (vir * m[a] * m[b] - (1.0 if a == b else 0.0))).sum()
    phi = np.fft.irfftn(S * th3 * C, s=(K3, K2, K1), axes=(0, 1, 2)) * (K1 * K2 * K3)
    dx, dy, dz = dtheta(wx, order), dtheta(wy, order), dtheta(wz, order)
    f = np.zeros((len(q), 3))
    for c in range(order):
        for b in range(order):
            g = phi[iz[:, c][:, None], iy[:, b][:, None], ix]          # [n, order] over x
            f[:, 0] += (dx * ty[:, b:b + 1] * tz[:, c:c + 1] * g).sum(1)
            f[:, 1] += (tx * dy[:, b:b + 1] * tz[:, c:c + 1] * g).sum(1)
            f[:, 2] += (tx * ty[:, b:b + 1] * dz[:, c:c + 1] * g).sum(1)
    g1 = -q * f[:, 0] * K1
    g2 = -q * f[:, 1] * K2
    g3 = -q * f[:, 2] * K3
    forces = g1[:, None] * R[0][None, :] + g2[:, None] * R[1][None, :] + g3[:, None] * R[2][None, :]
    return energy, W, forces


def self_energy(atoms, beta):
    q = np.asarray(atoms, dtype=np.float32)[:, 3].astype(np.float64)
    return -beta / np.sqrt(np.pi) * float((q * q).sum())


def ewald_recip_direct(pos, q, lattice, beta, tol=1e-14, chunk=256):
    """Direct Ewald reciprocal energy and forces (FP64), all m with
    exp(-pi^2 m^2 / beta^2) above tol."""
    R, vol = reciprocal(lattice)
    pos = np.asarray(pos, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    mmax = beta * np.sqrt(-np.log(tol)) / np.pi
    hmax = [int(np.ceil(mmax / np.linalg.norm(R[d]))) + 1 for d in range(3)]
    hs = np.array([(h, k, l) for h in range(0, hmax[0] + 1)
                   for k in range(-hmax[1], hmax[1] + 1)
                   for l in range(-hmax[2], hmax[2] + 1)
                   if (h, k, l) > (0, 0, 0) or h > 0], dtype=np.float64)
    # keep one of each +-m pair: h > 0, or h == 0 and (k, l) > (0, 0)
    keep = (hs[:, 0] > 0) | ((hs[:, 0] == 0) & ((hs[:, 1] > 0) | ((hs[:, 1] == 0) & (hs[:, 2] > 0))))
    hs = hs[keep]
    M = hs @ R
    msq = (M * M).sum(1)
    g = np.exp(-(np.pi ** 2) * msq / beta ** 2) / msq
    sel = g > tol / (mmax ** 2 + 1e-300)
    M, g = M[sel], g[sel]
    energy = 0.0
    forces = np.zeros_like(pos)
    for s in range(0, len(M), chunk):
        Mc, gc = M[s:s + chunk], g[s:s + chunk]
        ph = 2.0 * np.pi * (pos @ Mc.T)                       # [n, m]
        c, sn = np.cos(ph), np.sin(ph)
        Sr, Si = q @ c, q @ sn
        energy += 2.0 * (gc * (Sr * Sr + Si * Si)).sum()      # both +-m
        # F_j = (2/V) q_j sum_{all m} g m Im(S* e_j); +-m pairs give twice this
        im = c * Si[None, :] - sn * Sr[None, :]                # Im(e_j S*) * -1 ... sign below
        forces += (4.0 / vol) * q[:, None] * ((-im) * gc[None, :]) @ Mc
    energy /= (2.0 * np.pi * vol)
    return energy, forces
