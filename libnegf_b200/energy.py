"""Host side of the energy loop: the real-axis grid, the Fermi function and
the Landauer current integral, as libNEGF's integrations module has them.

- tunneling_int_def (src/integrations.F90:1613-1668): Npoints =
  nint((Emax - Emin) / Estep) + 1 points Emin + Estep*(i-1), every point
  weighted by kwght, dealt round robin over ranks (point i to rank
  mod(i-1, numprocs)).
- tunneling_and_dos (:1675-1783): tunn_mat(i, :) = T(E_i, pairs) * kwght
  and ldos_mat(i, :) = LDOS(E_i, sets) * kwght, summed over the k-points of
  the caller.
- fermi_f (src/distributions.F90:27-55), integrate_el (src/integrations.F90:
  2688-2770) and electron_current (:2430-2452): the current of pair ii =
  integrate_el(tunn_mat(:, ii), mu_ni, mu_nf, kT_ni, kT_nf) * g_spin.
"""
from __future__ import annotations

from typing import Dict, Optional, Sequence

import numpy as np

KB_HARTREE_PER_K = 3.166811389002312e-6   # Boltzmann constant in Hartree/K (src/ln_constants.F90)


def energy_grid(emin: float, emax: float, estep: float) -> np.ndarray:
    """tunneling_int_def: Npoints = nint((Emax-Emin)/Estep) + 1 real energies."""
    npts = int(np.rint((emax - emin) / estep)) + 1
    return emin + estep * np.arange(npts, dtype=np.float64)


def local_points(npts: int, rank: int = 0, world: int = 1) -> np.ndarray:
    """Indices (0-based) of the grid points rank `rank` solves: round robin."""
    return np.arange(rank, npts, world, dtype=np.int64)


def fermi_f(E, Ef: float, kT: float):
    """Fermi-Dirac occupation with the kT = 0 step and the |x| > 30 cut of
    fermi_f (src/distributions.F90:27-55)."""
    E = np.asarray(E, dtype=np.float64)
    if kT == 0.0:
        return np.where(E > Ef, 0.0, 1.0)
    x = (E - Ef) / kT
    out = np.empty_like(x)
    big = np.abs(x) > 30.0
    out[~big] = 1.0 / (np.exp(x[~big]) + 1.0)
    hi = big & (E > Ef)
    out[hi] = np.exp(-x[hi])
    out[big & ~hi] = 1.0
    return out


def integrate_el(tun, mu1: float, mu2: float, kT1: float, kT2: float, emin: float, emax: float, estep: float,
                 kb_1K: float = KB_HARTREE_PER_K) -> float:
    """integrate_el (src/integrations.F90:2688-2770): trapezoids of
    (f2 - f1) * T with T linearly interpolated on N sub-steps of each grid
    interval, N the first integer with step < (kT1 + kT2) / 20 (kT floored at
    1 K); the sign flips when mu2 < mu1 (the integral runs from the lower
    chemical potential)."""
    tun = np.asarray(tun, dtype=np.float64)
    npoints = int(np.rint((emax - emin) / estep))
    kbT1 = max(kT1, kb_1K)
    kbT2 = max(kT2, kb_1K)
    swapped = mu2 < mu1
    if swapped:
        mu1, mu2 = mu2, mu1
        kbT1, kbT2 = kbT2, kbT1
    # the sub-step count: the reference grows N from 1 until the sub-step is
    # below the threshold (it never resets N, and every interval has the
    # same width, so one N serves every interval)
    N = 0
    destep = 1.0e10
    curr = 0.0
    for i in range(npoints):
        E1 = emin + estep * i
        E2 = emin + estep * (i + 1)
        TT1, TT2 = tun[i], tun[i + 1]
        while destep >= (kbT1 + kbT2) / 20.0:
            N += 1
            destep = (E2 - E1) / N
        i1 = np.arange(N, dtype=np.float64)
        E3 = E1 + (E2 - E1) * i1 / N
        E4 = E3 + (E2 - E1) / N
        TT3 = (TT2 - TT1) * i1 / N + TT1
        TT4 = TT3 + (TT2 - TT1) / N
        c1 = (fermi_f(E3, mu2, kbT2) - fermi_f(E3, mu1, kbT1)) * TT3
        c2 = (fermi_f(E4, mu2, kbT2) - fermi_f(E4, mu1, kbT1)) * TT4
        # the reference accumulates sub-step by sub-step
        for v in (c1 + c2) * (E4 - E3) / 2.0:
            curr = curr + v
    return -curr if swapped else curr


def tunneling_and_dos(ctx, device_ids: Sequence[int], kweights: Sequence[float], emin: float, emax: float,
                      estep: float, pairs, eta: float = 1e-4, ldos: bool = False, dos_delta: float = 1e-4,
                      rank: int = 0, world: int = 1):
    """tunn_mat (Npoints x npairs) and, with ldos, ldos_mat (Npoints x nsets)
    over the k-points `device_ids` (uploaded devices) with weights kweights.
    Each rank solves its round-robin share of the grid in one batched call
    per k-point; rows of other ranks stay zero (the reference then reduces
    them across ranks).  Returns (E, tunn_mat, ldos_mat or None, status)."""
    E = energy_grid(emin, emax, estep)
    mine = local_points(E.size, rank, world)
    npairs = len(pairs)
    tunn = np.zeros((E.size, npairs))
    ldos_mat = None
    status = np.zeros(E.size, dtype=np.int32)
    for did, w in zip(device_ids, kweights):
        T, led, _, st = ctx.transmissions(did, E[mine], pairs, eta=eta, ldos=ldos, dos_delta=dos_delta)
        tunn[mine] += T * w
        if ldos:
            if ldos_mat is None:
                ldos_mat = np.zeros((E.size, led.shape[1]))
            ldos_mat[mine] += led * w
        status[mine] = np.where(status[mine] == 0, st, status[mine])
    return E, tunn, ldos_mat, status


def electron_current(tunn_mat, pairs, mu: Sequence[float], kT: Sequence[float], emin: float, emax: float,
                     estep: float, g_spin: float = 2.0, kb_1K: float = KB_HARTREE_PER_K) -> np.ndarray:
    """Current of every pair (electron_current, src/integrations.F90:2430-2452):
    integrate_el over tunn_mat(:, ii) between contacts ni and nf, times g_spin.
    mu and kT are per contact (1-based contact numbers in `pairs`)."""
    tunn_mat = np.asarray(tunn_mat, dtype=np.float64)
    out = np.zeros(len(pairs))
    for ii, (ni, nf) in enumerate(pairs):
        out[ii] = integrate_el(tunn_mat[:, ii], mu[ni - 1], mu[nf - 1], kT[ni - 1], kT[nf - 1], emin, emax,
                               estep, kb_1K) * g_spin
    return out
