"""NumPy twin of the CPU oracle (test infrastructure only).

An independent second restatement of the same reference routines, written
from the Fortran rather than from negf_oracle.cpp, used to catch
transcription errors in either.  np.linalg.inv is LAPACK zgesv
(= zgetrf + zgetrs on the identity, like zinv in src/inversions.F90:807-839)
and `@` is zgemm.  Pure Python loops: small cases only.
"""
from __future__ import annotations

import numpy as np

inv = np.linalg.inv


def dag(a):
    return a.conj().T


def spectral(s):
    """zspectral_dns: i (S - S^dag) (src/sparsekit_drv.F90:2870-2890)"""
    return 1j * (s - dag(s))


def decimation(Ao, Bo, Co, tol=1e-9, max_iter=300):
    """src/contselfenergy.F90:271-340"""
    Ao = Ao.copy(); Bo = Bo.copy(); Co = Co.copy()
    Ao_s = Ao.copy()
    ok = False
    ncyc = max_iter + 1
    for it in range(1, max_iter + 1):
        Go = inv(Ao)
        GoXCo = Go @ Co
        C1 = Co @ GoXCo
        if np.abs(C1).max() <= tol:
            if ok:
                ncyc = it
                break
            ok = True
        else:
            ok = False
        Self = Bo @ GoXCo
        Ao_s = Ao_s - Self
        Ao = Ao - Self
        GoXBo = Go @ Bo
        B1 = Bo @ GoXBo
        Ao = Ao - Co @ GoXBo
        Bo = B1
        Co = C1
    return inv(Ao_s), ncyc


def contact_sigma(dev, c, Ec, tol=1e-9, max_iter=300):
    """surface_green + compute_contacts_dns (src/contselfenergy.F90:184-207, 469-481)"""
    L = dev.lead_size[c]
    S00 = np.eye(L) if dev.lead_s00 is None else dev.lead_s00[c]
    S01 = np.zeros((L, L)) if dev.lead_s01 is None else dev.lead_s01[c]
    Ao = Ec * S00 - dev.lead_h00[c]
    Bo = Ec * S01 - dev.lead_h01[c]
    Co = dag(np.conj(Ec) * S01 - dev.lead_h01[c])
    gs, ncyc = decimation(Ao, Bo, Co, tol, max_iter)
    n0 = dev.surf(c)
    if n0 > 0:   # bound-surface block (src/contselfenergy.F90:226-243)
        SS = np.eye(n0 + L) if dev.lead_ss is None or dev.lead_ss[c] is None else dev.lead_ss[c]
        gt = Ec * SS - dev.lead_hs[c]
        gt[n0:, n0:] = inv(gs)
        gs = inv(gt)
    SMC = np.zeros_like(dev.hmc[c]) if dev.smc is None else dev.smc[c]
    Tlc = Ec * SMC - dev.hmc[c]
    Tcl = dag(np.conj(Ec) * SMC - dev.hmc[c])
    return Tlc @ gs @ Tcl, ncyc


def esh(dev, Ec, sig=None):
    """build_ESH (src/iterative.F90:1956-1982) as three block lists"""
    nbl = dev.nbl
    if dev.s_diag is None:
        d = [Ec * np.eye(b.shape[0]) - b for b in dev.h_diag]
        u = [-b for b in dev.h_upper]
        l = [-b for b in dev.h_lower]
    else:
        d = [Ec * s - h for s, h in zip(dev.s_diag, dev.h_diag)]
        u = [Ec * s - h for s, h in zip(dev.s_upper, dev.h_upper)]
        l = [Ec * s - h for s, h in zip(dev.s_lower, dev.h_lower)]
    if sig is not None:
        for c, cb in enumerate(dev.cblk):
            d[cb - 1] = d[cb - 1] - sig[c]
    return d, u, l


def gsmr(d, u, l):
    """calculate_gsmr_blocks(nbl -> 2, keep) (src/iterative_cpu.F90:51-124)"""
    nbl = len(d)
    g = [None] * nbl
    g[nbl - 1] = inv(d[nbl - 1])
    for i in range(nbl - 2, 0, -1):
        g[i] = inv(d[i] + (-(u[i] @ g[i + 1])) @ l[i])
    return g


def gr_blocks(d, u, l, g, upto=None):
    """Gr(1,1) then the tridiagonal sweep (src/iterative_cpu.F90:134-224)"""
    nbl = len(d)
    upto = nbl if upto is None else upto
    Gd = [None] * nbl
    Gl = [None] * (nbl - 1)
    Gu = [None] * (nbl - 1)
    if nbl == 1:
        Gd[0] = inv(d[0])
        return Gd, Gl, Gu
    Gd[0] = inv(d[0] - (u[0] @ g[1]) @ l[0])
    for k in range(1, upto):
        Gl[k - 1] = -((g[k] @ l[k - 1]) @ Gd[k - 1])
        w2 = u[k - 1] @ g[k]
        Gu[k - 1] = -(Gd[k - 1] @ w2)
        Gd[k] = g[k] + (-(Gl[k - 1] @ w2))
    return Gd, Gl, Gu


def transmission_2(ni, nf, sig, cblk, Gd):
    """src/iterative_cpu.F90:399-470"""
    ct1 = ni if cblk[ni - 1] < cblk[nf - 1] else nf
    G = Gd[cblk[ct1 - 1] - 1]
    gam = spectral(sig[ct1 - 1])
    trs = gam @ (1j * (G - dag(G))) - ((gam @ G) @ gam) @ dag(G)
    return abs(np.trace(trs).real)


def point_transmission(dev, E, eta=1e-4, ni=1, nf=2, tol=1e-9, max_iter=300):
    sig, ncyc = [], 0
    for c in range(dev.ncont):
        s, nc = contact_sigma(dev, c, E + 1j * eta, tol, max_iter)
        sig.append(s)
        ncyc = max(ncyc, nc)
    d, u, l = esh(dev, E + 0j, sig)
    g = gsmr(d, u, l)
    cb = dev.cblk
    if dev.ncont == 2 and min(cb[ni - 1], cb[nf - 1]) == 1:
        Gd, _, _ = gr_blocks(d, u, l, g, upto=1)
        return transmission_2(ni, nf, sig, cb, Gd), ncyc
    bl1, bl2 = sorted((cb[ni - 1], cb[nf - 1]))
    Gd, Gl, Gu = gr_blocks(d, u, l, g, upto=bl2)
    col = Gd[bl1 - 1]
    for i in range(bl1 + 1, bl2 + 1):
        col = Gl[i - 2] if i == bl1 + 1 else -(g[i - 1] @ l[i - 2]) @ col
    ct1, ct2 = (ni, nf) if cb[ni - 1] < cb[nf - 1] else (nf, ni)
    g1 = spectral(sig[ct1 - 1])
    g2 = spectral(sig[ct2 - 1])
    return abs(np.trace(((g2 @ col) @ g1) @ dag(col)).real), ncyc


def point_dos(dev, E, eta=1e-4, dos_delta=1e-4, ni=1, nf=2, tol=1e-9, max_iter=300):
    sig = [contact_sigma(dev, c, E + 1j * eta, tol, max_iter)[0] for c in range(dev.ncont)]
    d, u, l = esh(dev, E + 1j * dos_delta, sig)
    g = gsmr(d, u, l) if dev.nbl > 1 else [None]
    Gd, _, _ = gr_blocks(d, u, l, g)
    T = transmission_2(ni, nf, sig, dev.cblk, Gd) if dev.ncont == 2 else 0.0
    dos = np.concatenate([-np.diag(G).imag / np.pi for G in Gd])
    return T, dos
