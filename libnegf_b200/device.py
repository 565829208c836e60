"""Block-tridiagonal device description and its C-ABI packing.

A `Device` is libNEGF's device after `zcsr2blk_sod`
(src/sparsekit_drv.F90:3409-3436): the diagonal and first off-diagonal blocks
of H and S per principal layer (PL), plus, per contact, the blocks that
`extract_cont` (src/ln_extract.F90:37-75) hands to `surface_green`
(src/contselfenergy.F90:184-207) and to the contact self-energy
(src/contselfenergy.F90:469-481).  Blocks are complex128 numpy arrays; they
are packed column-major (the layout of `z_DNS%val`) into one contiguous
buffer per block family and described by the `negf_b200_device` C struct of
include/negf_b200.h.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_double_p = ctypes.POINTER(ctypes.c_double)


class NegfDeviceStruct(ctypes.Structure):
    """Mirror of `negf_b200_device` (include/negf_b200.h)."""

    _fields_ = [
        ("nbl", ctypes.c_int32),
        ("pl_size", c_int32_p),
        ("h_diag", c_double_p),
        ("h_upper", c_double_p),
        ("h_lower", c_double_p),
        ("s_diag", c_double_p),
        ("s_upper", c_double_p),
        ("s_lower", c_double_p),
        ("ncont", ctypes.c_int32),
        ("cblk", c_int32_p),
        ("lead_size", c_int32_p),
        ("lead_h00", c_double_p),
        ("lead_h01", c_double_p),
        ("lead_s00", c_double_p),
        ("lead_s01", c_double_p),
        ("hmc", c_double_p),
        ("smc", c_double_p),
        ("surf_size", c_int32_p),
        ("lead_hs", c_double_p),
        ("lead_ss", c_double_p),
    ]


def _pack(blocks: Optional[List[np.ndarray]]) -> Optional[np.ndarray]:
    if blocks is None:
        return None
    if len(blocks) == 0:
        return np.zeros(2, dtype=np.float64)
    flat = [np.asarray(b, dtype=np.complex128).ravel(order="F") for b in blocks]
    return np.ascontiguousarray(np.concatenate(flat)).view(np.float64)


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return c_double_p()
    return a.ctypes.data_as(c_double_p)


@dataclass
class Device:
    """Dense block-tridiagonal device with its contacts.

    h_diag[i]   H(i,i)    n_i x n_i
    h_upper[i]  H(i,i+1)  n_i x n_{i+1}
    h_lower[i]  H(i+1,i)  n_{i+1} x n_i
    s_* None    S = I
    cblk[c]     1-based device block of contact c (TStruct_info%cblk)
    lead_h00[c] contact PL1 on-site, lead_h01[c] contact PL1->PL2 coupling
    hmc[c]      device block cblk[c] -> contact PL1 coupling (n_cb x L_c)
    """

    h_diag: List[np.ndarray]
    h_upper: List[np.ndarray]
    h_lower: List[np.ndarray]
    cblk: List[int]
    lead_h00: List[np.ndarray]
    lead_h01: List[np.ndarray]
    hmc: List[np.ndarray]
    s_diag: Optional[List[np.ndarray]] = None
    s_upper: Optional[List[np.ndarray]] = None
    s_lower: Optional[List[np.ndarray]] = None
    lead_s00: Optional[List[np.ndarray]] = None
    lead_s01: Optional[List[np.ndarray]] = None
    smc: Optional[List[np.ndarray]] = None
    # bound surface layers (surfdim > 0): per contact n0 (0 = none) and, for
    # n0 > 0, H / S over Surf + PL1 ((n0 + L) x (n0 + L)); hmc / smc of such a
    # contact are n_cblk x (n0 + L)
    surf_size: Optional[List[int]] = None
    lead_hs: Optional[List[Optional[np.ndarray]]] = None
    lead_ss: Optional[List[Optional[np.ndarray]]] = None
    _keep: list = field(default_factory=list, repr=False)

    @property
    def nbl(self) -> int:
        return len(self.h_diag)

    @property
    def pl_size(self) -> List[int]:
        return [b.shape[0] for b in self.h_diag]

    @property
    def norb(self) -> int:
        return int(sum(self.pl_size))

    @property
    def ncont(self) -> int:
        return len(self.cblk)

    @property
    def lead_size(self) -> List[int]:
        return [b.shape[0] for b in self.lead_h00]

    def surf(self, c: int) -> int:
        return int(self.surf_size[c]) if self.surf_size is not None else 0

    def validate(self) -> None:
        n = self.pl_size
        nbl = self.nbl
        if nbl < 1:
            raise ValueError("device needs at least one principal layer")
        if len(self.h_upper) != nbl - 1 or len(self.h_lower) != nbl - 1:
            raise ValueError("need nbl-1 upper and lower coupling blocks")
        for i in range(nbl):
            if self.h_diag[i].shape != (n[i], n[i]):
                raise ValueError("H(%d,%d) has shape %s" % (i, i, self.h_diag[i].shape))
        for i in range(nbl - 1):
            if self.h_upper[i].shape != (n[i], n[i + 1]):
                raise ValueError("H(%d,%d) has shape %s" % (i, i + 1, self.h_upper[i].shape))
            if self.h_lower[i].shape != (n[i + 1], n[i]):
                raise ValueError("H(%d,%d) has shape %s" % (i + 1, i, self.h_lower[i].shape))
        if (self.s_diag is None) != (self.s_upper is None) or (self.s_diag is None) != (self.s_lower is None):
            raise ValueError("S blocks must be all given or all None")
        for c, cb in enumerate(self.cblk):
            if not 1 <= cb <= nbl:
                raise ValueError("cblk[%d]=%d outside 1..%d" % (c, cb, nbl))
            L = self.lead_h00[c].shape[0]
            if self.lead_h01[c].shape != (L, L):
                raise ValueError("lead_h01[%d] must be %dx%d" % (c, L, L))
            ngs = L + self.surf(c)
            if self.hmc[c].shape != (n[cb - 1], ngs):
                raise ValueError("hmc[%d] must be %dx%d" % (c, n[cb - 1], ngs))
            if self.surf(c) > 0:
                if self.lead_hs is None or self.lead_hs[c] is None or self.lead_hs[c].shape != (ngs, ngs):
                    raise ValueError("lead_hs[%d] must be %dx%d" % (c, ngs, ngs))
                if self.lead_ss is not None and self.lead_ss[c] is not None and self.lead_ss[c].shape != (ngs, ngs):
                    raise ValueError("lead_ss[%d] must be %dx%d" % (c, ngs, ngs))

    def to_struct(self) -> NegfDeviceStruct:
        """Packs the blocks; the returned struct references arrays kept alive
        by this object until the next call."""
        self.validate()
        keep = []

        def k(a):
            keep.append(a)
            return a

        pl = k(np.ascontiguousarray(self.pl_size, dtype=np.int32))
        cb = k(np.ascontiguousarray(self.cblk, dtype=np.int32))
        ls = k(np.ascontiguousarray(self.lead_size, dtype=np.int32))
        arrs = {}
        for name in ("h_diag", "h_upper", "h_lower", "s_diag", "s_upper", "s_lower",
                     "lead_h00", "lead_h01", "lead_s00", "lead_s01", "hmc", "smc"):
            arrs[name] = k(_pack(getattr(self, name))) if getattr(self, name) is not None else None
        st = NegfDeviceStruct()
        if self.surf_size is not None and any(self.surf(c) > 0 for c in range(self.ncont)):
            ss = k(np.ascontiguousarray([self.surf(c) for c in range(self.ncont)], dtype=np.int32))
            st.surf_size = ss.ctypes.data_as(c_int32_p)
            with_s = [c for c in range(self.ncont) if self.surf(c) > 0]
            st.lead_hs = _ptr(k(_pack([self.lead_hs[c] for c in with_s])))
            if self.lead_ss is not None and all(self.lead_ss[c] is not None for c in with_s):
                st.lead_ss = _ptr(k(_pack([self.lead_ss[c] for c in with_s])))
        st.nbl = self.nbl
        st.pl_size = pl.ctypes.data_as(c_int32_p)
        st.ncont = self.ncont
        st.cblk = cb.ctypes.data_as(c_int32_p)
        st.lead_size = ls.ctypes.data_as(c_int32_p)
        for name, a in arrs.items():
            setattr(st, name, _ptr(a))
        self._keep = keep
        return st

    def nbytes(self) -> int:
        tot = 0
        for name in ("h_diag", "h_upper", "h_lower", "s_diag", "s_upper", "s_lower",
                     "lead_h00", "lead_h01", "lead_s00", "lead_s01", "hmc", "smc"):
            v = getattr(self, name)
            if v is not None:
                tot += sum(b.size * 16 for b in v)
        return tot
