"""ctypes front-end of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product path never imports it.  See negf_oracle.cpp for the
reference routines each entry point restates.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from libnegf_b200.device import Device  # noqa: E402

_lib = None
KB_HARTREE_PER_K = 3.166811389002312e-6   # src/ln_constants.F90:36
KB_EV_PER_K = 8.617332411853536e-5        # src/ln_constants.F90:39


def lib():
    global _lib
    if _lib is None:
        from oracle import build as _b   # noqa: E402
        path = _b.build()
        L = ctypes.CDLL(path)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        vp = ctypes.c_void_p
        L.oracle_decimation.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_double, ctypes.c_int, dp, ip]
        L.oracle_zinv.argtypes = [ctypes.c_int, dp, dp]
        L.oracle_decimation_xp.argtypes = [ctypes.c_int, dp, dp, dp, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_int, dp, ip]
        L.oracle_transmission.argtypes = [vp, ctypes.c_int, dp, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_int, ctypes.c_double, dp, ip, ip, ctypes.c_int]
        L.oracle_transmission_dos.argtypes = [vp, ctypes.c_int, dp, ctypes.c_double, ctypes.c_double,
                                              ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                              ctypes.c_double, dp, dp, ip, ip, ctypes.c_int]
        L.oracle_meir_wingreen.argtypes = [vp, ctypes.c_int, dp, ctypes.c_double, dp, dp, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                           dp, dp, dp, ip, dp, ip, ip, ctypes.c_int]
        L.oracle_transmissions.argtypes = [vp, ctypes.c_int, dp, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                           ip, ip, vp, ctypes.c_int, ip, ip, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_double, dp, dp, ip, ip, ctypes.c_int]
        L.oracle_density.argtypes = [vp, ctypes.c_int, dp, dp, dp, ctypes.c_double, ctypes.c_int, dp, dp, dp, dp, dp,
                                     ip, ip, ctypes.c_int]
        L.oracle_density_neq.argtypes = [vp, ctypes.c_int, dp, ctypes.c_double, dp, dp, dp, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_int, dp, dp, dp, dp, dp, ip, ip,
                                         ctypes.c_int]
        L.oracle_transmission_xp.argtypes = [vp, ctypes.c_int, dp, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, ctypes.c_int, ctypes.c_int, dp, dp, ip, ip,
                                             ctypes.c_int]
        L.oracle_fermi.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.oracle_fermi.restype = ctypes.c_double
        L.oracle_integrate_el.argtypes = [dp, ctypes.c_int] + [ctypes.c_double] * 8
        L.oracle_integrate_el.restype = ctypes.c_double
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _i(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _flatF(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.complex128).ravel(order="F"))


def decimation(Ao, Bo, Co, tol=1e-9, max_iter=300):
    n = Ao.shape[0]
    a, b, c = (_flatF(x) for x in (Ao, Bo, Co))
    g = np.zeros(n * n, dtype=np.complex128)
    ncyc = np.zeros(1, dtype=np.int32)
    st = lib().oracle_decimation(n, _d(a.view(np.float64)), _d(b.view(np.float64)), _d(c.view(np.float64)),
                                 tol, max_iter, _d(g.view(np.float64)), _i(ncyc))
    return g.reshape((n, n), order="F"), int(ncyc[0]), st


def decimation_xp(Ao, Bo, Co, tol=1e-9, max_iter=300, extended=True, gauss_jordan=False):
    """decimation restated over long double (extended) or over double with its
    own unblocked LU (or Gauss-Jordan) inverses and triple-loop products."""
    n = Ao.shape[0]
    a, b, c = (_flatF(x) for x in (Ao, Bo, Co))
    g = np.zeros(n * n, dtype=np.complex128)
    ncyc = np.zeros(1, dtype=np.int32)
    st = lib().oracle_decimation_xp(n, _d(a.view(np.float64)), _d(b.view(np.float64)), _d(c.view(np.float64)),
                                    tol, max_iter, 1 if extended else (2 if gauss_jordan else 0),
                                    _d(g.view(np.float64)), _i(ncyc))
    return g.reshape((n, n), order="F"), int(ncyc[0]), st


def zinv(A):
    n = A.shape[0]
    a = _flatF(A)
    x = np.zeros(n * n, dtype=np.complex128)
    st = lib().oracle_zinv(n, _d(a.view(np.float64)), _d(x.view(np.float64)))
    return x.reshape((n, n), order="F"), st


def transmission(dev: Device, energies, eta=1e-4, ni=1, nf=2, sgf_tol=1e-9, sgf_max_iter=300,
                 eps=0.0, nthreads=0):
    E = np.ascontiguousarray(energies, dtype=np.float64)
    npts = E.size
    T = np.zeros(npts)
    ncyc = np.zeros(npts, dtype=np.int32)
    status = np.zeros(npts, dtype=np.int32)
    st = dev.to_struct()
    lib().oracle_transmission(ctypes.addressof(st), npts, _d(E), eta, ni, nf, sgf_tol, sgf_max_iter, eps,
                              _d(T), _i(ncyc), _i(status), nthreads)
    return T, ncyc, status


def transmission_xp(dev: Device, energies, eta=1e-4, dos_delta=None, sgf_tol=1e-9, sgf_max_iter=300,
                    extended=True, nthreads=0, gauss_jordan=False):
    """The 2-contact T path (dos_delta None) or T + DOS path restated over
    long double (extended=True: 64-bit significand, a near-exact solution of
    the same algorithm) or over double with its own unblocked LU and
    triple-loop products (extended=False: a second FP64 rounding path; with
    gauss_jordan=True the inverses are Gauss-Jordan eliminations instead).
    Returns T, dos (or None), ncyc, status."""
    E = np.ascontiguousarray(energies, dtype=np.float64)
    npts = E.size
    T = np.zeros(npts)
    dos = np.zeros((npts, dev.norb)) if dos_delta is not None else None
    ncyc = np.zeros(npts, dtype=np.int32)
    status = np.zeros(npts, dtype=np.int32)
    st = dev.to_struct()
    rc = lib().oracle_transmission_xp(ctypes.addressof(st), npts, _d(E), eta,
                                      0.0 if dos_delta is None else dos_delta, sgf_tol, sgf_max_iter,
                                      1 if extended else (2 if gauss_jordan else 0), _d(T),
                                      _d(dos) if dos is not None else None,
                                      _i(ncyc), _i(status), nthreads)
    if rc != 0:
        raise ValueError("oracle_transmission_xp: status %d (two contacts only)" % rc)
    return T, dos, ncyc, status


def transmission_dos(dev: Device, energies, eta=1e-4, dos_delta=1e-4, ni=1, nf=2, sgf_tol=1e-9,
                     sgf_max_iter=300, eps=0.0, nthreads=0):
    E = np.ascontiguousarray(energies, dtype=np.float64)
    npts = E.size
    T = np.zeros(npts)
    dos = np.zeros((npts, dev.norb))
    ncyc = np.zeros(npts, dtype=np.int32)
    status = np.zeros(npts, dtype=np.int32)
    st = dev.to_struct()
    lib().oracle_transmission_dos(ctypes.addressof(st), npts, _d(E), eta, dos_delta, ni, nf, sgf_tol,
                                  sgf_max_iter, eps, _d(T), _d(dos), _i(ncyc), _i(status), nthreads)
    return T, dos, ncyc, status


def transmissions(dev: Device, energies, pairs, eta=1e-4, tun_proj=None, dos_proj=None, dos_delta=0.0,
                  sgf_tol=1e-9, sgf_max_iter=300, eps=0.0, nthreads=0):
    """calculate_transmissions (dos_proj None) or calculate_transmissions_and_dos
    over contact pairs [(ni, nf), ...]; tun_proj: 1-based orbital indices;
    dos_proj: list of 1-based index lists.  Returns T (npts x npairs), ledos
    (npts x nsets or None), ncyc, status."""
    from libnegf_b200.projections import tun_mask, dos_sets
    E = np.ascontiguousarray(energies, dtype=np.float64)
    npts = E.size
    ni = np.ascontiguousarray([p[0] for p in pairs], dtype=np.int32)
    nf = np.ascontiguousarray([p[1] for p in pairs], dtype=np.int32)
    npairs = ni.size
    T = np.zeros((npts, npairs))
    mask = tun_mask(dev.norb, tun_proj)
    mask_p = mask.ctypes.data if mask is not None else None
    if dos_proj is not None:
        ptr, idx = dos_sets(dos_proj)
        nsets = ptr.size - 1
        ledos = np.zeros((npts, max(nsets, 1)))
    else:
        ptr = np.zeros(1, dtype=np.int32)
        idx = np.zeros(1, dtype=np.int32)
        nsets = 0
        ledos = None
    ncyc = np.zeros(npts, dtype=np.int32)
    status = np.zeros(npts, dtype=np.int32)
    st = dev.to_struct()
    lib().oracle_transmissions(ctypes.addressof(st), npts, _d(E), eta, dos_delta, npairs, _i(ni), _i(nf), mask_p,
                               nsets, _i(ptr), _i(idx), sgf_tol, sgf_max_iter, eps, _d(T),
                               _d(ledos) if ledos is not None else None, _i(ncyc), _i(status), nthreads)
    return T, (ledos[:, :nsets] if ledos is not None else None), ncyc, status


def density(dev: Device, z, w, sgf_tol=1e-9, sgf_max_iter=300, nthreads=0):
    """contour_int over complex points z with complex weights w: the density
    matrix blocks (lists of diag, upper, lower blocks), ncyc, status."""
    z = np.ascontiguousarray(z, dtype=np.complex128).ravel()
    wt = np.ascontiguousarray(w, dtype=np.complex128).ravel()
    er = np.ascontiguousarray(z.real)
    ei = np.ascontiguousarray(z.imag)
    n = dev.pl_size
    nd = sum(x * x for x in n)
    no = sum(n[i] * n[i + 1] for i in range(len(n) - 1))
    rd = np.zeros(max(nd, 1), dtype=np.complex128)
    ru = np.zeros(max(no, 1), dtype=np.complex128)
    rl = np.zeros(max(no, 1), dtype=np.complex128)
    nm = sum(n[cb - 1] * L for cb, L in zip(dev.cblk, dev.lead_size))
    rdc = np.zeros(max(nm, 1), dtype=np.complex128)
    rcd = np.zeros(max(nm, 1), dtype=np.complex128)
    ncyc = np.zeros(z.size, dtype=np.int32)
    status = np.zeros(z.size, dtype=np.int32)
    st = dev.to_struct()
    lib().oracle_density(ctypes.addressof(st), z.size, _d(er), _d(ei), _d(wt.view(np.float64)), sgf_tol,
                         sgf_max_iter, _d(rd.view(np.float64)), _d(ru.view(np.float64)), _d(rl.view(np.float64)),
                         _d(rdc.view(np.float64)), _d(rcd.view(np.float64)), _i(ncyc), _i(status), nthreads)
    from libnegf_b200.density import split_blocks, split_outer
    return split_blocks(n, rd, ru, rl), split_outer(dev, rdc, rcd), ncyc, status


def density_neq(dev: Device, energies, w, frm, eta=1e-4, coupling=None, scba_niter=5, scba_tol=1e-7,
                sgf_tol=1e-9, sgf_max_iter=300, nthreads=0):
    """real_axis_int: sum_p w_p Gn(E_p) blocks, the calculate_Gn_outer
    blocks per contact (device->contact, contact->device), ncyc, status."""
    E = np.ascontiguousarray(energies, dtype=np.float64).ravel()
    wt = np.ascontiguousarray(w, dtype=np.complex128).ravel()
    f = np.ascontiguousarray(frm, dtype=np.float64)
    cp = None if coupling is None else np.ascontiguousarray(coupling, dtype=np.float64)
    n = dev.pl_size
    nd = sum(x * x for x in n)
    no = sum(n[i] * n[i + 1] for i in range(len(n) - 1))
    rd = np.zeros(max(nd, 1), dtype=np.complex128)
    ru = np.zeros(max(no, 1), dtype=np.complex128)
    rl = np.zeros(max(no, 1), dtype=np.complex128)
    nm = sum(n[cb - 1] * L for cb, L in zip(dev.cblk, dev.lead_size))
    rdc = np.zeros(max(nm, 1), dtype=np.complex128)
    rcd = np.zeros(max(nm, 1), dtype=np.complex128)
    ncyc = np.zeros(E.size, dtype=np.int32)
    status = np.zeros(E.size, dtype=np.int32)
    st = dev.to_struct()
    lib().oracle_density_neq(ctypes.addressof(st), E.size, _d(E), eta, _d(wt.view(np.float64)), _d(f),
                             _d(cp) if cp is not None else None, scba_niter, scba_tol, sgf_tol, sgf_max_iter,
                             _d(rd.view(np.float64)), _d(ru.view(np.float64)), _d(rl.view(np.float64)),
                             _d(rdc.view(np.float64)), _d(rcd.view(np.float64)), _i(ncyc), _i(status), nthreads)
    from libnegf_b200.density import split_blocks, split_outer
    return split_blocks(n, rd, ru, rl), split_outer(dev, rdc, rcd), ncyc, status


def meir_wingreen(dev: Device, energies, frm, coupling=None, eta=1e-4, scba_niter=5, scba_tol=1e-7,
                  sgf_tol=1e-9, sgf_max_iter=300, eps=0.0, nthreads=0, scba_mix=1.0, scba_rule=0):
    """meir_wingreen + layer_current with the elastic SCBA per point.  The
    defaults are the reference rule (no mixing, max |dGn| < scba_tol);
    scba_mix < 1 mixes the dephasing self-energies linearly from zero and
    scba_rule = 1 stops on the change of the contact-1 current instead."""
    E = np.ascontiguousarray(energies, dtype=np.float64)
    npts = E.size
    frm = np.ascontiguousarray(np.broadcast_to(frm, (npts, dev.ncont)), dtype=np.float64)
    cp = None if coupling is None else np.ascontiguousarray(np.broadcast_to(coupling, (dev.norb,)),
                                                             dtype=np.float64)
    curr = np.zeros((npts, dev.ncont))
    lcurr = np.zeros((npts, max(dev.nbl - 1, 1)))
    ldens = np.zeros((npts, dev.nbl))
    it = np.zeros(npts, dtype=np.int32)
    err = np.zeros(npts)
    ncyc = np.zeros(npts, dtype=np.int32)
    status = np.zeros(npts, dtype=np.int32)
    st = dev.to_struct()
    lib().oracle_meir_wingreen(ctypes.addressof(st), npts, _d(E), eta, _d(frm),
                               _d(cp) if cp is not None else ctypes.POINTER(ctypes.c_double)(),
                               scba_niter, scba_tol, scba_mix, scba_rule, sgf_tol, sgf_max_iter, eps,
                               _d(curr), _d(lcurr), _d(ldens), _i(it), _d(err), _i(ncyc), _i(status), nthreads)
    return dict(curr=curr, layer_curr=lcurr[:, :dev.nbl - 1], layer_dens=ldens, scba_iter=it,
                scba_err=err, ncyc=ncyc, status=status)


def fermi(E, Ef, kT):
    return lib().oracle_fermi(E, Ef, kT)


def integrate_el(tun, mu1, mu2, kT1, kT2, emin, emax, estep, kb_1K=KB_HARTREE_PER_K):
    t = np.ascontiguousarray(tun, dtype=np.float64)
    return lib().oracle_integrate_el(_d(t), t.size, mu1, mu2, kT1, kT2, emin, emax, estep, kb_1K)
