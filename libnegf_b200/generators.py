"""Seeded synthetic devices.

libNEGF publishes no benchmark inputs and its test inputs are git-LFS files
absent from the reference tree, so every workload here is generated from a
seed.  The generators follow the workload definitions of the transport
benchmarks this package is measured on:

  transport_c0  N=20 PLs, n=32, orthogonal tight binding: random Hermitian
                on-site blocks (diagonal U[-1,1] eV, off-diagonal complex
                Gaussian sigma=0.1), inter-layer couplings complex Gaussian
                sigma=0.3 rescaled so the lead band spans about +-3 eV, S=I.
                Leads repeat the first / last layer.
  transport_c1  N=100, n=256 nanowire: blocks with 10 % random non-zeros
                (sigma=0.2), on-site disorder U[-0.5,0.5] eV,
                S = I + 0.05*(random Hermitian, same sparsity); transverse
                k enters as a Bloch phase on per-layer transverse couplings.
  transport_c2  the c1 generator at N=60, n=512.
  transport_c3  the c0 generator at N=40, n=128 (dephasing SCBA workload).
  chain         perfect 1-D chain (analytic known answers: T=1 in band).

Contact convention (contselfenergy.F90:184-207): the contact's PL1 touches
the device, PL2 continues away from it; `hmc` couples device block cblk to
PL1, `lead_h01` couples PL1 to PL2.  A lead that "repeats" a device layer
with rightward coupling U has PL1->PL2 coupling U for a right lead and
U^dagger for a left lead.
"""
from __future__ import annotations

from typing import List, Optional, Sequence

import numpy as np

from .device import Device


def _cgauss(rng, shape, sigma):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * (sigma / np.sqrt(2.0))


def _herm_onsite(rng, n, sigma_off, diag_lo, diag_hi, density=1.0):
    z = _cgauss(rng, (n, n), sigma_off)
    if density < 1.0:
        z = z * (rng.random((n, n)) < density)
    up = np.triu(z, 1)
    h = up + up.conj().T
    h = h + np.diag(rng.uniform(diag_lo, diag_hi, n))
    return h.astype(np.complex128)


def chain(n_per_pl: int = 1, nbl: int = 4, t: float = 1.0, eps0: float = 0.0,
          cblk: Sequence[int] = None) -> Device:
    """Perfect 1-D chain, hopping -t, on-site eps0; band eps0 +- 2t.

    Each PL holds `n_per_pl` consecutive sites; both leads are the same chain.
    """
    m = n_per_pl
    H0 = np.zeros((m, m), np.complex128)
    for i in range(m):
        H0[i, i] = eps0
        if i + 1 < m:
            H0[i, i + 1] = H0[i + 1, i] = -t
    V = np.zeros((m, m), np.complex128)   # PL j -> PL j+1 (rightward)
    V[m - 1, 0] = -t
    if cblk is None:
        cblk = [1, nbl]
    hd = [H0.copy() for _ in range(nbl)]
    hu = [V.copy() for _ in range(nbl - 1)]
    hl = [V.conj().T.copy() for _ in range(nbl - 1)]
    lead_h00, lead_h01, hmc = [], [], []
    for cb in cblk:
        lead_h00.append(H0.copy())
        if cb == 1:      # left lead: device block 1 -> PL1 is leftward
            hmc.append(V.conj().T.copy())
            lead_h01.append(V.conj().T.copy())
        else:            # right lead
            hmc.append(V.copy())
            lead_h01.append(V.copy())
    return Device(hd, hu, hl, list(cblk), lead_h00, lead_h01, hmc)


def _attach_leads(hd, hu, hl, sd, su, sl, cblk_order):
    """Leads that repeat the first / last layer with the adjacent coupling."""
    nbl = len(hd)
    lead_h00, lead_h01, hmc = [], [], []
    lead_s00, lead_s01, smc = [], [], []
    for cb in cblk_order:
        if cb == 1:
            U = hu[0]                # layer 1 -> 2 (rightward) of the device
            lead_h00.append(hd[0].copy())
            lead_h01.append(U.conj().T.copy())
            hmc.append(U.conj().T.copy())
            if sd is not None:
                Us = su[0]
                lead_s00.append(sd[0].copy())
                lead_s01.append(Us.conj().T.copy())
                smc.append(Us.conj().T.copy())
        else:
            U = hu[nbl - 2]
            lead_h00.append(hd[nbl - 1].copy())
            lead_h01.append(U.copy())
            hmc.append(U.copy())
            if sd is not None:
                Us = su[nbl - 2]
                lead_s00.append(sd[nbl - 1].copy())
                lead_s01.append(Us.copy())
                smc.append(Us.copy())
    if sd is None:
        return lead_h00, lead_h01, hmc, None, None, None
    return lead_h00, lead_h01, hmc, lead_s00, lead_s01, smc


def transport_c0(nbl: int = 20, n: int = 32, seed: int = 0,
                 cblk: Sequence[int] = None, bandwidth: float = 3.0) -> Device:
    """Orthogonal tight-binding device (the c0 generator; also c3 at N=40,
    n=128).  Uniform PL size n; S = I."""
    rng = np.random.default_rng(seed)
    hd = [_herm_onsite(rng, n, 0.1, -1.0, 1.0) for _ in range(nbl)]
    V = [_cgauss(rng, (n, n), 0.3) for _ in range(max(nbl - 1, 1))]
    # rescale all couplings so that ||H_1|| + 2 ||V_1|| = bandwidth
    h1 = np.linalg.norm(hd[0], 2)
    v1 = np.linalg.norm(V[0], 2)
    s = max(bandwidth - h1, 0.5) / (2.0 * v1)
    # the 2-norms come from LAPACK, whose last bits depend on the host CPU's
    # kernels: quantise the scale so the device is bit-identical everywhere
    s = float(np.round(s * 2.0 ** 24) / 2.0 ** 24)
    V = [s * v for v in V]
    hu = [V[i].copy() for i in range(nbl - 1)]
    hl = [V[i].conj().T.copy() for i in range(nbl - 1)]
    if nbl == 1:
        hu, hl = [], []
        # single-layer device: leads couple through V[0]
    if cblk is None:
        cblk = [1, nbl]
    if nbl == 1:
        U = V[0]
        lead_h00 = [hd[0].copy(), hd[0].copy()]
        lead_h01 = [U.conj().T.copy(), U.copy()]
        hmc = [U.conj().T.copy(), U.copy()]
        return Device(hd, hu, hl, list(cblk), lead_h00, lead_h01, hmc)
    lh00, lh01, hmc, _, _, _ = _attach_leads(hd, hu, hl, None, None, None, cblk)
    return Device(hd, hu, hl, list(cblk), lh00, lh01, hmc)


def transport_c1(nbl: int = 100, n: int = 256, seed: int = 1, kpoint: float = 0.0,
                 density: float = 0.1, sigma: float = 0.2, disorder: float = 0.5,
                 s_scale: float = 0.05, cblk: Sequence[int] = None) -> Device:
    """Sparse nanowire-like device with non-orthogonal overlap (the c1/c2
    generator).  `kpoint` is the transverse Bloch phase k (radians): each
    layer's on-site block gets T_i e^{ik} + T_i^dag e^{-ik} from a per-layer
    transverse coupling T_i.  The random draws depend only on `seed`, so all
    k-points of one device share the same structure."""
    rng = np.random.default_rng(seed)
    hd, hu, hl, sd, su, sl = [], [], [], [], [], []
    ph = np.exp(1j * kpoint)
    for i in range(nbl):
        h = _herm_onsite(rng, n, sigma, -disorder, disorder, density)
        T = _cgauss(rng, (n, n), sigma) * (rng.random((n, n)) < density)
        h = h + T * ph + T.conj().T * np.conj(ph)
        hd.append(h)
        r = _herm_onsite(rng, n, sigma, -sigma, sigma, density)
        sd.append(np.eye(n, dtype=np.complex128) + s_scale * r)
    for i in range(nbl - 1):
        V = _cgauss(rng, (n, n), sigma) * (rng.random((n, n)) < density)
        R = _cgauss(rng, (n, n), sigma) * (V != 0)
        hu.append(V)
        hl.append(V.conj().T.copy())
        su.append(s_scale * R)
        sl.append(s_scale * R.conj().T)
    if cblk is None:
        cblk = [1, nbl]
    lh00, lh01, hmc, ls00, ls01, smc = _attach_leads(hd, hu, hl, sd, su, sl, cblk)
    return Device(hd, hu, hl, list(cblk), lh00, lh01, hmc,
                  s_diag=sd, s_upper=su, s_lower=sl,
                  lead_s00=ls00, lead_s01=ls01, smc=smc)


def uneven(pl_sizes: Sequence[int], seed: int = 3, cblk: Sequence[int] = None) -> Device:
    """Orthogonal device with uneven PL sizes (grouped-tile coverage).  The
    leads repeat the first / last layer."""
    rng = np.random.default_rng(seed)
    nbl = len(pl_sizes)
    hd = [_herm_onsite(rng, m, 0.1, -1.0, 1.0) for m in pl_sizes]
    hu, hl = [], []
    for i in range(nbl - 1):
        V = _cgauss(rng, (pl_sizes[i], pl_sizes[i + 1]), 0.3) * 0.5
        hu.append(V)
        hl.append(V.conj().T.copy())
    if cblk is None:
        cblk = [1, nbl]
    # leads need square PL couplings: use an on-site-sized lead coupling
    lead_h00, lead_h01, hmc = [], [], []
    for cb in cblk:
        m = pl_sizes[cb - 1]
        U = _cgauss(rng, (m, m), 0.3) * 0.5
        lead_h00.append(hd[cb - 1].copy())
        lead_h01.append(U if cb != 1 else U.conj().T.copy())
        hmc.append(U if cb != 1 else U.conj().T.copy())
    return Device(hd, hu, hl, list(cblk), lead_h00, lead_h01, hmc)


def energy_grid(emin: float, emax: float, npts: int) -> np.ndarray:
    """Uniform grid Emin + Estep*(i-1), i = 1..Npoints, as tunneling_int_def
    builds it (src/integrations.F90:1617-1633)."""
    if npts == 1:
        return np.array([emin], dtype=np.float64)
    estep = (emax - emin) / (npts - 1)
    return emin + estep * np.arange(npts, dtype=np.float64)


def band_edge_energies(dev: Device, contact: int = 0, nk: int = 64, n_edges: int = 64,
                       window: float = 1e-3, seed: int = 7) -> np.ndarray:
    """Energies clustered within `window` of the band edges of one lead
    (periodic PL chain H00 + H01 e^{ik} + h.c., S = I part only)."""
    h00 = dev.lead_h00[contact]
    h01 = dev.lead_h01[contact]
    ks = np.linspace(0.0, np.pi, nk)
    edges = []
    for k in ks:
        h = h00 + h01 * np.exp(1j * k) + h01.conj().T * np.exp(-1j * k)
        ev = np.linalg.eigvalsh(h)
        edges.append(ev)
    ev = np.array(edges)
    band_min = ev.min(axis=0)
    band_max = ev.max(axis=0)
    pts = np.sort(np.concatenate([band_min, band_max]))
    rng = np.random.default_rng(seed)
    sel = pts[rng.integers(0, len(pts), n_edges)]
    return np.sort(sel + rng.uniform(-window, window, n_edges))


def transport_c1_kpoints(kpoints: Sequence[float], nbl: int = 100, n: int = 256, seed: int = 1,
                         density: float = 0.1, sigma: float = 0.2, disorder: float = 0.5,
                         s_scale: float = 0.05, cblk: Sequence[int] = None) -> List[Device]:
    """transport_c1 at several transverse k-points.  The k-independent blocks
    (couplings, overlap) are drawn once and shared between the returned
    devices; only the on-site blocks (and the lead on-site blocks that
    repeat them) carry the Bloch phase.  Device k equals transport_c1(...,
    kpoint=k) with the same seed."""
    rng = np.random.default_rng(seed)
    H0, T, sd = [], [], []
    for i in range(nbl):
        H0.append(_herm_onsite(rng, n, sigma, -disorder, disorder, density))
        T.append(_cgauss(rng, (n, n), sigma) * (rng.random((n, n)) < density))
        r = _herm_onsite(rng, n, sigma, -sigma, sigma, density)
        sd.append(np.eye(n, dtype=np.complex128) + s_scale * r)
    hu, hl, su, sl = [], [], [], []
    for i in range(nbl - 1):
        V = _cgauss(rng, (n, n), sigma) * (rng.random((n, n)) < density)
        R = _cgauss(rng, (n, n), sigma) * (V != 0)
        hu.append(V)
        hl.append(V.conj().T.copy())
        su.append(s_scale * R)
        sl.append(s_scale * R.conj().T)
    if cblk is None:
        cblk = [1, nbl]
    out = []
    for k in kpoints:
        ph = np.exp(1j * k)
        hd = [H0[i] + T[i] * ph + T[i].conj().T * np.conj(ph) for i in range(nbl)]
        lh00, lh01, hmc, ls00, ls01, smc = _attach_leads(hd, hu, hl, sd, su, sl, cblk)
        out.append(Device(hd, hu, hl, list(cblk), lh00, lh01, hmc, s_diag=sd, s_upper=su, s_lower=sl,
                          lead_s00=ls00, lead_s01=ls01, smc=smc))
    return out


def with_periodic_surface(dev: Device, contact: int, layers: int = 1) -> Device:
    """The same device with `layers` principal layers of contact `contact`
    moved into a bound surface block (surfdim = layers * L): the contact's
    region becomes Surf | PL1 | PL2 with Surf made of periodic copies of the
    lead PL.  The surface Green's function of Surf + PL1 then restricts to the
    lead's own surface GF on Surf, so every result equals the original
    device's (a known answer for the bound-surface block)."""
    import copy
    d = copy.deepcopy(dev)
    c = contact
    L = d.lead_h00[c].shape[0]
    n0 = layers * L
    ngs = n0 + L
    H00, H01 = d.lead_h00[c], d.lead_h01[c]
    S00 = None if d.lead_s00 is None else d.lead_s00[c]
    S01 = None if d.lead_s01 is None else d.lead_s01[c]
    nl = layers + 1   # surface layers + PL1
    hs = np.zeros((ngs, ngs), np.complex128)
    ss = np.zeros((ngs, ngs), np.complex128)
    for k in range(nl):
        sl = slice(k * L, (k + 1) * L)
        hs[sl, sl] = H00
        ss[sl, sl] = np.eye(L) if S00 is None else S00
        if k + 1 < nl:
            nx = slice((k + 1) * L, (k + 2) * L)
            hs[sl, nx] = H01
            hs[nx, sl] = H01.conj().T
            if S01 is not None:
                ss[sl, nx] = S01
                ss[nx, sl] = S01.conj().T
    hmc = np.zeros((d.hmc[c].shape[0], ngs), np.complex128)
    hmc[:, :L] = d.hmc[c]
    d.hmc[c] = hmc
    if d.smc is not None:
        smc = np.zeros_like(hmc)
        smc[:, :L] = d.smc[c]
        d.smc[c] = smc
    d.surf_size = [0] * d.ncont if d.surf_size is None else list(d.surf_size)
    d.surf_size[c] = n0
    d.lead_hs = [None] * d.ncont if d.lead_hs is None else list(d.lead_hs)
    d.lead_hs[c] = hs
    if S00 is not None or S01 is not None:
        d.lead_ss = [None] * d.ncont if d.lead_ss is None else list(d.lead_ss)
        d.lead_ss[c] = ss
    return d
