"""Device description from a global sparse H (and S), as libNEGF builds it.

libNEGF takes the whole Hamiltonian in CSR (negf_set_h / negf_set_s,
src/api/libnegf_api.f90) plus the block structure of negf_init_structure
(:146-185, create_TStruct src/ln_structure.F90:77-145):

- plend(1..npl): last orbital of every principal layer (PL) of the device;
- per contact: surfstart, surfend (a surface block, empty when
  surfend = surfstart - 1), contend (last orbital of the contact's two PLs);
- cblk: the device PL each contact couples to.

The per-energy solve then reads dense blocks: the tridiagonal device blocks
of ES - H (zcsr2blk_sod, src/sparsekit_drv.F90:3409-3436), and per contact
HC/SC over the contact's two PLs and HMC/SMC between the cblk PL and the
contact's first PL (extract_cont, src/ln_extract.F90:37-75).  This module
does that extraction once per k on the host and returns the Device the
C-ABI uploads; E enters on the device.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np

from .device import Device


def _dense(M, r0, r1, c0, c1):
    """M[r0:r1, c0:c1] (0-based, end exclusive) as a dense complex128 block."""
    blk = M[r0:r1, c0:c1]
    if hasattr(blk, "toarray"):
        blk = blk.toarray()
    return np.ascontiguousarray(np.asarray(blk, dtype=np.complex128))


def device_from_csr(H, S, plend: Sequence[int], cblk: Sequence[int], surfstart: Sequence[int],
                    surfend: Sequence[int], contend: Sequence[int]) -> Device:
    """Blocks of H (and S; None = identity, as negf_set_s_id) for the
    structure of negf_init_structure (1-based indices).  H and S may be
    scipy.sparse matrices or dense arrays over device + contact orbitals.
    A contact with surface orbitals (surfend >= surfstart: libNEGF's
    surfdim = surfend - surfstart + 1 > 0, Surf | PL1 | PL2) gets its bound
    surface block (H and S over Surf + PL1, the block surface_green inverts,
    src/contselfenergy.F90:226-243) and a coupling to Surf + PL1."""
    plend = [int(x) for x in plend]
    npl = len(plend)
    if npl < 1:
        raise ValueError("need at least one principal layer")
    starts = [0] + plend[:-1]                      # 0-based first orbital of each PL
    if any(plend[i] <= starts[i] for i in range(npl)):
        raise ValueError("plend must increase")
    ncont = len(cblk)
    if not (len(surfstart) == len(surfend) == len(contend) == ncont):
        raise ValueError("surfstart, surfend, contend and cblk need one entry per contact")
    hd = [_dense(H, starts[i], plend[i], starts[i], plend[i]) for i in range(npl)]
    hu = [_dense(H, starts[i], plend[i], starts[i + 1], plend[i + 1]) for i in range(npl - 1)]
    hl = [_dense(H, starts[i + 1], plend[i + 1], starts[i], plend[i]) for i in range(npl - 1)]
    if S is not None:
        sd = [_dense(S, starts[i], plend[i], starts[i], plend[i]) for i in range(npl)]
        su = [_dense(S, starts[i], plend[i], starts[i + 1], plend[i + 1]) for i in range(npl - 1)]
        sl = [_dense(S, starts[i + 1], plend[i + 1], starts[i], plend[i]) for i in range(npl - 1)]
    else:
        sd = su = sl = None
    lh00, lh01, hmc = [], [], []
    ls00, ls01, smc = [], [], []
    surf, lhs, lss = [], [], []
    for c in range(ncont):
        b0, c_start, c_end = int(surfstart[c]), int(surfend[c]) + 1, int(contend[c])
        n0 = c_start - b0                            # surfdim
        if n0 < 0:
            raise ValueError("contact %d: surfend < surfstart - 1" % (c + 1))
        nd = c_end - c_start + 1                     # the two periodic PLs
        if nd < 2 or nd % 2:
            raise ValueError("contact %d: its two PLs must have equal size (dimension %d)" % (c + 1, nd))
        L = nd // 2
        j0 = b0 - 1                                  # 0-based first orbital of the contact (surface first)
        p1 = j0 + n0                                 # 0-based first orbital of PL1
        ngs = n0 + L
        lh00.append(_dense(H, p1, p1 + L, p1, p1 + L))
        lh01.append(_dense(H, p1, p1 + L, p1 + L, p1 + 2 * L))
        cb = int(cblk[c])
        if not 1 <= cb <= npl:
            raise ValueError("cblk[%d] = %d outside 1..%d" % (c, cb, npl))
        hmc.append(_dense(H, starts[cb - 1], plend[cb - 1], j0, j0 + ngs))
        surf.append(n0)
        lhs.append(_dense(H, j0, j0 + ngs, j0, j0 + ngs) if n0 > 0 else None)
        lss.append(_dense(S, j0, j0 + ngs, j0, j0 + ngs) if (n0 > 0 and S is not None) else None)
        if S is not None:
            ls00.append(_dense(S, p1, p1 + L, p1, p1 + L))
            ls01.append(_dense(S, p1, p1 + L, p1 + L, p1 + 2 * L))
            smc.append(_dense(S, starts[cb - 1], plend[cb - 1], j0, j0 + ngs))
    any_surf = any(n > 0 for n in surf)
    dev = Device(hd, hu, hl, [int(x) for x in cblk], lh00, lh01, hmc,
                 s_diag=sd, s_upper=su, s_lower=sl,
                 lead_s00=ls00 if S is not None else None, lead_s01=ls01 if S is not None else None,
                 smc=smc if S is not None else None,
                 surf_size=surf if any_surf else None, lead_hs=lhs if any_surf else None,
                 lead_ss=lss if (any_surf and S is not None) else None)
    dev.validate()
    return dev


def csr_arrays(H, S=None):
    """The arrays negf_b200_upload_csr takes: 1-based rowptr / colind (int32)
    of one pattern, and the complex values of H and of S (or None) on it.
    With S, the pattern is the union of both sparsity patterns, each matrix
    holding zeros where only the other has an entry."""
    import scipy.sparse as sp
    H = sp.csr_matrix(H, dtype=np.complex128)
    if S is None:
        H = H.copy()
        H.sum_duplicates()
        return (np.ascontiguousarray(H.indptr + 1, dtype=np.int32), np.ascontiguousarray(H.indices + 1, dtype=np.int32),
                np.ascontiguousarray(H.data), None)
    S = sp.csr_matrix(S, dtype=np.complex128)
    if S.shape != H.shape:
        raise ValueError("H and S differ in shape")
    pattern = (abs(H) + abs(S)).tocsr()
    pattern.sum_duplicates()
    pattern.sort_indices()
    rows = np.repeat(np.arange(pattern.shape[0]), np.diff(pattern.indptr))
    hv = np.ascontiguousarray(np.asarray(H[rows, pattern.indices]).ravel(), dtype=np.complex128)
    sv = np.ascontiguousarray(np.asarray(S[rows, pattern.indices]).ravel(), dtype=np.complex128)
    return (np.ascontiguousarray(pattern.indptr + 1, dtype=np.int32),
            np.ascontiguousarray(pattern.indices + 1, dtype=np.int32), hv, sv)


def csr_from_device(dev: Device):
    """The inverse layout (for tests and examples): the global sparse H (and
    S, or None) of a Device with its contacts appended after the device
    orbitals, two PLs each, and the negf_init_structure arrays.  Returns
    (H, S, plend, cblk, surfstart, surfend, contend)."""
    import scipy.sparse as sp
    n = dev.pl_size
    norb = dev.norb
    plend = list(np.cumsum(n))
    starts = [0] + plend[:-1]
    L = dev.lead_size
    n0s = [dev.surf(c) for c in range(dev.ncont)]
    ntot = norb + sum(2 * L[c] + n0s[c] for c in range(dev.ncont))
    H = sp.lil_matrix((ntot, ntot), dtype=np.complex128)
    S = sp.lil_matrix((ntot, ntot), dtype=np.complex128) if dev.s_diag is not None else None
    for i in range(dev.nbl):
        H[starts[i]:plend[i], starts[i]:plend[i]] = dev.h_diag[i]
        if S is not None:
            S[starts[i]:plend[i], starts[i]:plend[i]] = dev.s_diag[i]
    for i in range(dev.nbl - 1):
        H[starts[i]:plend[i], starts[i + 1]:plend[i + 1]] = dev.h_upper[i]
        H[starts[i + 1]:plend[i + 1], starts[i]:plend[i]] = dev.h_lower[i]
        if S is not None:
            S[starts[i]:plend[i], starts[i + 1]:plend[i + 1]] = dev.s_upper[i]
            S[starts[i + 1]:plend[i + 1], starts[i]:plend[i]] = dev.s_lower[i]
    surfstart, surfend, contend = [], [], []
    off = norb
    for c in range(dev.ncont):
        l, n0 = L[c], n0s[c]
        j0 = off
        p1 = j0 + n0                                  # first orbital of PL1 (after the surface)
        surfstart.append(j0 + 1)
        surfend.append(j0 + n0)
        contend.append(j0 + n0 + 2 * l)
        H[p1:p1 + l, p1:p1 + l] = dev.lead_h00[c]
        H[p1 + l:p1 + 2 * l, p1 + l:p1 + 2 * l] = dev.lead_h00[c]
        H[p1:p1 + l, p1 + l:p1 + 2 * l] = dev.lead_h01[c]
        H[p1 + l:p1 + 2 * l, p1:p1 + l] = dev.lead_h01[c].conj().T
        if n0 > 0:
            H[j0:p1 + l, j0:p1 + l] = dev.lead_hs[c]
        cb = dev.cblk[c]
        H[starts[cb - 1]:plend[cb - 1], j0:p1 + l] = dev.hmc[c]
        H[j0:p1 + l, starts[cb - 1]:plend[cb - 1]] = dev.hmc[c].conj().T
        if S is not None:
            s00 = dev.lead_s00[c] if dev.lead_s00 is not None else np.eye(l)
            s01 = dev.lead_s01[c] if dev.lead_s01 is not None else np.zeros((l, l))
            smc = dev.smc[c] if dev.smc is not None else np.zeros((n[cb - 1], n0 + l))
            S[p1:p1 + l, p1:p1 + l] = s00
            S[p1 + l:p1 + 2 * l, p1 + l:p1 + 2 * l] = s00
            S[p1:p1 + l, p1 + l:p1 + 2 * l] = s01
            S[p1 + l:p1 + 2 * l, p1:p1 + l] = s01.conj().T
            if n0 > 0:
                S[j0:p1 + l, j0:p1 + l] = (dev.lead_ss[c] if dev.lead_ss is not None and dev.lead_ss[c] is not None
                                           else np.eye(n0 + l))
            S[starts[cb - 1]:plend[cb - 1], j0:p1 + l] = smc
            S[j0:p1 + l, starts[cb - 1]:plend[cb - 1]] = smc.conj().T
        off += n0 + 2 * l
    return (H.tocsr(), S.tocsr() if S is not None else None, plend, list(dev.cblk), surfstart, surfend, contend)
