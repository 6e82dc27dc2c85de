"""FP64 smooth-PME reciprocal-space restatement -- TEST INFRASTRUCTURE.

ProtoMol has no PME: its only Ewald reciprocal term is the explicit k-sum
of NonbondedFullEwaldSystemForce::reciprocalTerm
(force/nonbonded/NonbondedFullEwaldSystemForce.h:868-1083), with energy
E = (4 pi / V) sum_{half space k} exp(-k^2 / 4 a^2) / k^2 |S(k)|^2.
This module restates the smooth particle-mesh Ewald approximation of that
same sum (Essmann, Perera, Berkowitz, Darden, Lee, Pedersen, J. Chem. Phys.
103, 8577 (1995)): cardinal B-spline charge spreading (order p), a 3-D FFT,
the influence function exp(-pi^2 m^2 / a^2) / (pi V m^2) |b(m)|^2 and force
gathering from the B-spline derivatives.  The GPU PME is checked against
this at matched grid, order and alpha; this restatement is in turn checked
to converge to the reference's k-sum as the grid is refined and the order
raised (tests/test_oracle_pins.py).
"""
from __future__ import annotations

import numpy as np


def bspline(fr: np.ndarray, p: int):
    """M_p(fr + k) and dM_p/du for k = 0..p-1 (Cox-de Boor recursion)."""
    n = fr.shape[0]
    m = np.zeros((n, p))
    m[:, 0] = fr
    m[:, 1] = 1.0 - fr
    dm = None
    for order in range(3, p + 1):
        if order == p:
            dm = m.copy()
            dm[:, 1:] -= m[:, :-1]
        new = np.zeros_like(m)
        prev = np.zeros(n)
        for k in range(order):
            cur = m[:, k] if k < order - 1 else np.zeros(n)
            x = fr + k
            new[:, k] = (x * cur + (order - x) * prev) / (order - 1)
            prev = cur
        m = new
    if p == 2:
        dm = np.stack([np.ones(n), -np.ones(n)], 1)
    return m, dm


def bspline_moduli(K: int, p: int) -> np.ndarray:
    """|b(m)|^2 = 1 / |sum_{k=0}^{p-2} M_p(k+1) exp(2 pi i m k / K)|^2."""
    mk, _ = bspline(np.zeros(1), p)  # M_p(k) at integers k = 0..p-1
    mk = mk[0]
    m = np.arange(K)
    s = np.zeros(K, dtype=complex)
    for k in range(p - 1):
        s += mk[k + 1] * np.exp(2j * np.pi * m * k / K)
    mod = np.abs(s) ** 2
    for i in range(K):
        if mod[i] < 1e-7:
            mod[i] = 0.5 * (mod[(i - 1) % K] + mod[(i + 1) % K])
    return 1.0 / mod


def reciprocal(pos: np.ndarray, charge: np.ndarray, box, alpha: float, p: int, K):
    """SPME reciprocal forces (n,3) and energy for an orthogonal box.
    box: edge length, 3 edges, or the 12-value (e1,e2,e3,origin) array."""
    box = np.asarray(box, dtype=np.float64).reshape(-1)
    if box.size == 12:
        Ls = np.array([box[0], box[4], box[8]])
        lo = box[9:12] - 0.5 * Ls
    else:
        Ls = np.broadcast_to(box, (3,)).astype(np.float64)
        lo = -0.5 * Ls
    Ks = np.broadcast_to(np.asarray(K), (3,)).astype(int)
    n = len(charge)
    frac = (pos - lo) / Ls
    frac -= np.floor(frac)
    u = frac * Ks
    iu = np.floor(u).astype(int)
    fr = u - iu
    iu %= Ks
    th, dth = [], []
    for a in range(3):
        t, d = bspline(fr[:, a], p)
        th.append(t)
        dth.append(d)
    ks = np.arange(p)
    gx = (iu[:, 0:1] - ks) % Ks[0]
    gy = (iu[:, 1:2] - ks) % Ks[1]
    gz = (iu[:, 2:3] - ks) % Ks[2]
    Q = np.zeros(tuple(Ks))
    w = charge[:, None, None, None] * th[0][:, :, None, None] * th[1][:, None, :, None] * \
        th[2][:, None, None, :]
    ix = np.broadcast_to(gx[:, :, None, None], w.shape)
    iy = np.broadcast_to(gy[:, None, :, None], w.shape)
    iz = np.broadcast_to(gz[:, None, None, :], w.shape)
    np.add.at(Q, (ix.ravel(), iy.ravel(), iz.ravel()), w.ravel())
    V = float(np.prod(Ls))
    m = [np.fft.fftfreq(int(Ks[a]), d=1.0 / Ks[a]) for a in range(3)]
    hx, hy, hz = np.meshgrid(m[0] / Ls[0], m[1] / Ls[1], m[2] / Ls[2], indexing="ij")
    h2 = hx * hx + hy * hy + hz * hz
    h2[0, 0, 0] = 1.0
    B = bspline_moduli(int(Ks[0]), p)[:, None, None] * bspline_moduli(int(Ks[1]), p)[None, :, None] \
        * bspline_moduli(int(Ks[2]), p)[None, None, :]
    G = np.exp(-np.pi ** 2 * h2 / alpha ** 2) / (np.pi * V * h2) * B
    G[0, 0, 0] = 0.0
    FQ = np.fft.fftn(Q)
    energy = 0.5 * float(np.sum(G * np.abs(FQ) ** 2))
    phi = np.real(np.fft.ifftn(G * FQ)) * Q.size
    vals = phi[ix, iy, iz]
    fx = -(charge * Ks[0] / Ls[0]) * np.einsum("na,nb,nc,nabc->n", dth[0], th[1], th[2], vals)
    fy = -(charge * Ks[1] / Ls[1]) * np.einsum("na,nb,nc,nabc->n", th[0], dth[1], th[2], vals)
    fz = -(charge * Ks[2] / Ls[2]) * np.einsum("na,nb,nc,nabc->n", th[0], th[1], dth[2], vals)
    return np.stack([fx, fy, fz], 1), energy
