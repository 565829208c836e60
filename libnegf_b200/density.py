"""Equilibrium density matrix by contour integration.

contour_int_def (src/integrations.F90:675-835) places the points of the
integral of Gr(z) f(z) in the complex plane: a Gauss-Legendre arc of Np_n(1)
points from the lower energy bound Elow, a second arc (kT = 0) or a segment
parallel to the real axis (kT > 0) of Np_n(2) points, and n_poles Fermi
poles mu + i pi kT (2k - 1).  contour_int (:844-897) sums w_p Gr(z_p) and
takes rho = i (T - T^dag); negf_b200_density does that sum on the device for
the tridiagonal blocks, and blk2csr (src/iterative.F90:1375-1450) keeps the
entries on the sparsity of S, here `restrict_to_pattern`.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np


def gauleg(x1: float, x2: float, n: int) -> Tuple[np.ndarray, np.ndarray]:
    """Gauss-Legendre nodes and weights on [x1, x2] in the order and with the
    sign convention of gauleg (src/integrations.F90:1468-1526): nodes run
    from x1 towards x2, weights carry the sign of x2 - x1."""
    t, W = np.polynomial.legendre.leggauss(n)
    xm, xl = 0.5 * (x2 + x1), 0.5 * (x2 - x1)
    return xm + xl * t, xl * W


def fermi_c(z, Ef: float, kT: float):
    """fermi_fc (src/distributions.F90:77-111) of a complex energy."""
    z = np.asarray(z, dtype=np.complex128)
    if kT == 0.0:
        return np.where(z.real > Ef, 0.0 + 0.0j, 1.0 + 0.0j)
    x = (z.real - Ef) / kT
    out = np.empty_like(z)
    big = np.abs(x) > 30.0
    hi = big & (z.real > Ef)
    out[hi] = np.exp(-(z[hi] - Ef) / kT)
    out[big & ~hi] = 1.0
    out[~big] = 1.0 / (np.exp((z[~big] - Ef) / kT) + 1.0)
    return out


def contour_points(elow: float, muref: float, kT: float, n_kt: float, np1: int, np2: int, n_poles: int,
                   g_spin: float = 2.0) -> Tuple[np.ndarray, np.ndarray]:
    """Points and weights of contour_int_def for the equilibrium case (no
    inelastic interaction): returns (z, w), complex arrays of length
    np1 + np2 + n_poles."""
    pi = np.pi
    nkT = n_kt * kT
    mumin = muref - nkT
    lam = 2.0 * n_poles * kT * pi if n_poles else 0.5 * kT * pi
    centre = (lam ** 2 - elow ** 2 + mumin ** 2) / (2.0 * (mumin - elow))
    rad = centre - elow
    alpha = 0.1 * pi if kT == 0.0 else np.arctan(lam / (mumin - centre))
    zs, ws = [], []
    p, wg = gauleg(pi, alpha, np1)
    Pc = rad * np.exp(1j * p)
    zs.append(centre + Pc)
    ws.append(1j * Pc * g_spin * wg / (2.0 * pi))
    if kT == 0.0:
        p, wg = gauleg(alpha, 0.0, np2)
        Pc = rad * np.exp(1j * p)
        zs.append(centre + Pc)
        ws.append((g_spin * wg / (2.0 * pi)) * Pc * 1j)
    else:
        z1 = muref + nkT + 1j * lam
        z2 = muref - nkT + 1j * lam
        zd = z2 - z1
        p, wg = gauleg(1.0, 0.0, np2)
        Ec = z1 + p * zd
        zs.append(Ec)
        ws.append(g_spin * zd * fermi_c(Ec, muref, kT) * wg / (2.0 * pi))
    k = np.arange(1, n_poles + 1)
    zs.append(muref + 1j * kT * pi * (2.0 * k - 1.0))
    ws.append(np.full(n_poles, -1j * g_spin * kT))
    return np.concatenate(zs).astype(np.complex128), np.concatenate(ws).astype(np.complex128)


def real_axis_points(mu: Sequence[float], kT: Sequence[float], n_kt: float, np_real: int, delta: float,
                     g_spin: float = 2.0) -> Tuple[np.ndarray, np.ndarray]:
    """real_axis_int_def (src/integrations.F90:989-1084), elastic case:
    np_real Gauss-Legendre energies on [min mu - Omega, max mu + Omega],
    Omega = n_kt * max kT, weights g_spin w / (2 pi).  Returns (E, w); the
    contacts see E + i*delta."""
    omega = n_kt * max(kT)
    x, wg = gauleg(min(mu) - omega, max(mu) + omega, np_real)
    return x, (g_spin * wg / (2.0 * np.pi)).astype(np.complex128)


def neq_occupations(E, mu: Sequence[float], kT: Sequence[float], ref: int) -> np.ndarray:
    """f_c(E) - f_ref(E) per point and contact (ref is 1-based): the
    occupations calculate_Gn_neq_components folds into Sigma^n."""
    from .energy import fermi_f
    E = np.asarray(E, dtype=np.float64)
    f = np.stack([fermi_f(E, m, t) for m, t in zip(mu, kT)], axis=1)
    return np.ascontiguousarray(f - f[:, ref - 1:ref])


def split_blocks(pl: Sequence[int], diag, upper, lower):
    """Flat block arrays (the h_diag / h_upper / h_lower layout) -> lists of
    column-major blocks (diag, upper, lower)."""
    pl = list(pl)
    d, u, l = [], [], []
    o = 0
    for n in pl:
        d.append(np.asarray(diag[o:o + n * n]).reshape((n, n), order="F"))
        o += n * n
    o = 0
    for i in range(len(pl) - 1):
        n, m = pl[i], pl[i + 1]
        u.append(np.asarray(upper[o:o + n * m]).reshape((n, m), order="F"))
        l.append(np.asarray(lower[o:o + n * m]).reshape((m, n), order="F"))
        o += n * m
    return d, u, l


def split_outer(dev, dc, cd):
    """Flat outer blocks (hmc layout) -> per contact (device->contact n_cb x L,
    contact->device L x n_cb)."""
    out_dc, out_cd = [], []
    o = 0
    for cb, L in zip(dev.cblk, dev.lead_size):
        n = dev.pl_size[cb - 1]
        out_dc.append(np.asarray(dc[o:o + n * L]).reshape((n, L), order="F"))
        out_cd.append(np.asarray(cd[o:o + n * L]).reshape((L, n), order="F"))
        o += n * L
    return out_dc, out_cd


def restrict_to_pattern(blocks, pattern, plend: Sequence[int]):
    """blk2csr: the entries of the tridiagonal blocks on the sparsity of
    `pattern` (a scipy.sparse matrix over at least the device orbitals);
    entries outside the device rows / columns or the tridiagonal are left
    out.  Returns a scipy CSR matrix of the device size."""
    import scipy.sparse as sp
    d, u, l = blocks
    plend = [int(x) for x in plend]
    starts = [0] + plend[:-1]
    norb = plend[-1]
    P = sp.csr_matrix(pattern)[:norb, :norb].tocoo()
    blk = np.searchsorted(np.asarray(plend), np.arange(norb), side="right")
    bi, bj = blk[P.row], blk[P.col]
    vals = np.zeros(P.nnz, dtype=np.complex128)
    for q in range(P.nnz):
        x, y = bi[q], bj[q]
        r, c = P.row[q] - starts[x], P.col[q] - starts[y]
        if x == y:
            vals[q] = d[x][r, c]
        elif y == x + 1:
            vals[q] = u[x][r, c]
        elif y == x - 1:
            vals[q] = l[y][r, c]
    return sp.csr_matrix((vals, (P.row, P.col)), shape=(norb, norb))


def density_matrix(ctx, device_id, z, w, pl: Sequence[int]):
    """Contour sum on the device (negf_b200_density): the density-matrix
    blocks (diag, upper, lower lists), ncyc and status per point."""
    return ctx.density(device_id, z, w, pl)
