"""ctypes binding of libnegf_b200.so (the C-ABI of include/negf_b200.h).

The CUDA extension is the only implementation: there is no CPU fallback.
Importing this module without a built libnegf_b200.so raises, and creating a
context without a GPU raises NegfError(NO_GPU).
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

from .device import Device
from .projections import dos_sets, tun_indices

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnegf_b200.so")

OK, SINGULAR, NOT_CONVERGED, NONFINITE, NOMEM, BAD_ARG, CUDA, TIMEOUT, ADMISSION, NO_GPU = range(10)
SCBA_NOT_CONVERGED = 10
# codes that concern the whole call (nothing was solved): raised even with check=False, which
# only lets per-point codes (SINGULAR, NOT_CONVERGED, NONFINITE, TIMEOUT, ...) through
CALL_ERRORS = (BAD_ARG, NOMEM, CUDA, ADMISSION, NO_GPU)
STATUS_NAMES = {0: "OK", 1: "SINGULAR", 2: "NOT_CONVERGED", 3: "NONFINITE", 4: "NOMEM", 5: "BAD_ARG",
                6: "CUDA", 7: "TIMEOUT", 8: "ADMISSION", 9: "NO_GPU", 10: "SCBA_NOT_CONVERGED"}

# every symbol include/negf_b200.h declares
EXPORTED = [
    "negf_b200_default_options", "negf_b200_version", "negf_b200_ctx_create", "negf_b200_ctx_destroy",
    "negf_b200_set_options", "negf_b200_last_error", "negf_b200_upload_device", "negf_b200_release_device",
    "negf_b200_device_bytes", "negf_b200_transmission", "negf_b200_transmission_dos",
    "negf_b200_meir_wingreen", "negf_b200_transmission_dev", "negf_b200_transmission_dos_dev",
    "negf_b200_zgemm_batched", "negf_b200_zinv_work_bytes", "negf_b200_zinv_batched",
    "negf_b200_decimation_work_bytes", "negf_b200_decimation_batched", "negf_b200_set_tracing",
    "negf_b200_get_trace", "negf_b200_decimation_noalloc", "negf_b200_set_tun_proj", "negf_b200_set_dos_proj",
    "negf_b200_transmissions", "negf_b200_set_sgf_cache", "negf_b200_sgf_cache_stats",
    "negf_b200_set_workspace_limit", "negf_b200_density", "negf_b200_density_neq", "negf_b200_meir_wingreen_dev",
    "negf_b200_sgf_cache_save", "negf_b200_sgf_cache_load", "negf_b200_upload_csr",
    "negf_b200_zgemm_i8_work_bytes", "negf_b200_zgemm_batched_i8", "negf_b200_launch_count",
]
TRACE_PHASES = ["gemm", "inv_panel", "inv_update", "inv_other", "elementwise", "total", "points", "unused"]


class DeviceShape:
    """Structure of a device uploaded from CSR (its blocks live only on the
    GPU): what the solve wrappers need to size their outputs."""

    def __init__(self, pl_size, cblk, lead_size):
        self.pl_size = list(pl_size)
        self.cblk = list(cblk)
        self.lead_size = list(lead_size)

    nbl = property(lambda self: len(self.pl_size))
    norb = property(lambda self: int(sum(self.pl_size)))
    ncont = property(lambda self: len(self.cblk))


class NegfError(RuntimeError):
    def __init__(self, code: int, msg: str = ""):
        self.code = code
        super().__init__("%s (%d)%s" % (STATUS_NAMES.get(code, "?"), code, (": " + msg) if msg else ""))


class Options(ctypes.Structure):
    """Mirror of negf_b200_options."""
    _fields_ = [("sgf_tol", ctypes.c_double), ("sgf_max_iter", ctypes.c_int32), ("eps_drop", ctypes.c_double),
                ("scba_tol", ctypes.c_double), ("scba_niter", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("ctas_per_sm", ctypes.c_int32), ("scba_mix", ctypes.c_double), ("scba_rule", ctypes.c_int32),
                ("schedule", ctypes.c_int32)]


_lib = None


def load():
    """Loads the extension; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libnegf_b200.so is not built (run __graft_entry__.build() or "
                          "python libnegf_b200/build.py); there is no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)
    i32, f64 = ctypes.c_int32, ctypes.c_double
    L.negf_b200_version.restype = ctypes.c_char_p
    L.negf_b200_last_error.restype = ctypes.c_char_p
    L.negf_b200_last_error.argtypes = [vp]
    L.negf_b200_default_options.argtypes = [ctypes.POINTER(Options)]
    L.negf_b200_ctx_create.argtypes = [i32, ctypes.POINTER(vp)]
    L.negf_b200_ctx_destroy.argtypes = [vp]
    L.negf_b200_set_options.argtypes = [vp, ctypes.POINTER(Options)]
    L.negf_b200_upload_device.argtypes = [vp, vp, ip]
    L.negf_b200_upload_csr.argtypes = [vp, i32, i32, ip, ip, dp, dp, i32, ip, i32, ip, ip, ip, ip, ip]
    L.negf_b200_release_device.argtypes = [vp, i32]
    L.negf_b200_device_bytes.argtypes = [vp, i32, ctypes.POINTER(ctypes.c_size_t)]
    L.negf_b200_transmission.argtypes = [vp, i32, ip, dp, f64, i32, i32, dp, ip, ip]
    L.negf_b200_transmission_dos.argtypes = [vp, i32, ip, dp, f64, f64, i32, i32, dp, dp, ip, ip]
    L.negf_b200_meir_wingreen.argtypes = [vp, i32, ip, dp, f64, dp, dp, dp, dp, dp, ip, dp, ip, ip]
    L.negf_b200_transmission_dev.argtypes = [vp, i32, vp, vp, f64, i32, i32, vp, vp, vp, vp]
    L.negf_b200_transmission_dos_dev.argtypes = [vp, i32, vp, vp, f64, f64, i32, i32, vp, vp, ctypes.c_int64,
                                                 vp, vp, vp]
    L.negf_b200_meir_wingreen_dev.argtypes = [vp, i32, vp, vp, f64, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32, i32, vp]
    L.negf_b200_zgemm_batched.argtypes = [i32, i32, i32, i32, dp, vp, ctypes.c_int64, vp, ctypes.c_int64, dp, vp,
                                          ctypes.c_int64, i32, vp]
    L.negf_b200_zgemm_i8_work_bytes.restype = ctypes.c_size_t
    L.negf_b200_zgemm_i8_work_bytes.argtypes = [i32, i32, i32, i32, i32]
    L.negf_b200_zgemm_batched_i8.argtypes = [i32, i32, i32, i32, dp, vp, ctypes.c_int64, vp, ctypes.c_int64, dp,
                                             vp, ctypes.c_int64, i32, vp, vp, vp]
    L.negf_b200_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
    L.negf_b200_zinv_work_bytes.restype = ctypes.c_size_t
    L.negf_b200_zinv_work_bytes.argtypes = [i32, i32]
    L.negf_b200_zinv_batched.argtypes = [i32, i32, vp, vp, vp, vp, vp]
    L.negf_b200_decimation_work_bytes.restype = ctypes.c_size_t
    L.negf_b200_decimation_work_bytes.argtypes = [i32, i32]
    L.negf_b200_decimation_batched.argtypes = [i32, i32, vp, vp, vp, vp, vp, f64, i32, vp, vp]
    L.negf_b200_set_tracing.argtypes = [vp, i32]
    L.negf_b200_get_trace.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
    L.negf_b200_decimation_noalloc.argtypes = [i32, i32, vp, vp, vp, vp, vp, f64, i32, vp]
    L.negf_b200_set_tun_proj.argtypes = [vp, i32, i32, ip]
    L.negf_b200_set_dos_proj.argtypes = [vp, i32, i32, ip, ip]
    L.negf_b200_transmissions.argtypes = [vp, i32, ip, dp, f64, f64, i32, ip, ip, dp, dp, ip, ip]
    L.negf_b200_set_sgf_cache.argtypes = [vp, i32, ctypes.c_size_t]
    L.negf_b200_set_workspace_limit.argtypes = [vp, ctypes.c_size_t]
    L.negf_b200_density.argtypes = [vp, i32, i32, dp, dp, dp, dp, dp, dp, dp, dp, ip, ip]
    L.negf_b200_density_neq.argtypes = [vp, i32, i32, dp, f64, dp, dp, dp, dp, dp, dp, dp, dp, ip, ip]
    i64p = ctypes.POINTER(ctypes.c_int64)
    L.negf_b200_sgf_cache_stats.argtypes = [vp, i64p, i64p, i64p, ctypes.POINTER(ctypes.c_size_t)]
    L.negf_b200_sgf_cache_save.argtypes = [vp, ctypes.c_char_p, i64p]
    L.negf_b200_sgf_cache_load.argtypes = [vp, ctypes.c_char_p, i64p]
    _lib = L
    return L


def _d(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else ctypes.POINTER(ctypes.c_double)()


def _i(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) if a is not None else ctypes.POINTER(ctypes.c_int32)()


class Context:
    """One CUDA device, its stream, the HBM-resident device descriptions and
    the persistent-kernel workspace (negf_b200_ctx)."""

    def __init__(self, cuda_device: int = 0, **options):
        L = load()
        h = ctypes.c_void_p()
        rc = L.negf_b200_ctx_create(cuda_device, ctypes.byref(h))
        if rc != OK:
            raise NegfError(rc, "negf_b200_ctx_create")
        self._h = h
        self._L = L
        self.devices = {}
        self._nldos = {}
        self.options = {}
        if options:
            self.set_options(**options)

    # -- lifecycle
    def close(self):
        if getattr(self, "_h", None):
            self._L.negf_b200_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def last_error(self) -> str:
        return self._L.negf_b200_last_error(self._h).decode()

    def _check(self, rc, what):
        if rc not in (OK,):
            raise NegfError(rc, "%s: %s" % (what, self.last_error()))

    def set_options(self, **kw):
        """The library defaults (negf_b200_default_options) with `kw` on top."""
        o = Options()
        self._L.negf_b200_default_options(ctypes.byref(o))
        for k, v in kw.items():
            if not hasattr(o, k):
                raise TypeError("unknown option %s" % k)
            setattr(o, k, v)
        self._check(self._L.negf_b200_set_options(self._h, ctypes.byref(o)), "set_options")
        self.options = dict(kw)

    def update_options(self, **kw):
        """The options set so far with `kw` on top."""
        self.set_options(**{**self.options, **kw})

    def launch_count(self) -> int:
        """Kernels this context's solve calls have launched so far."""
        c = ctypes.c_uint64()
        self._check(self._L.negf_b200_launch_count(self._h, ctypes.byref(c)), "launch_count")
        return int(c.value)

    def set_tracing(self, enable=True):
        self._check(self._L.negf_b200_set_tracing(self._h, 1 if enable else 0), "set_tracing")

    def get_trace(self) -> dict:
        """Per-phase SM cycles summed over CTAs since the last call (reset)."""
        buf = (ctypes.c_uint64 * 8)()
        self._check(self._L.negf_b200_get_trace(self._h, buf), "get_trace")
        return {k: int(v) for k, v in zip(TRACE_PHASES, buf)}

    def upload(self, dev: Device) -> int:
        st = dev.to_struct()
        did = ctypes.c_int32()
        self._check(self._L.negf_b200_upload_device(self._h, ctypes.byref(st), ctypes.byref(did)), "upload")
        self.devices[did.value] = dev
        return did.value

    def upload_csr(self, H, S, plend, cblk, surfstart, surfend, contend) -> int:
        """Uploads a device from the global sparse H (and S, or None for
        S = I) and the negf_init_structure arrays (1-based), the blocks
        being extracted on the GPU (negf_b200_upload_csr).  H and S go to
        the C-ABI on their union pattern."""
        from .structure import csr_arrays
        rp, ci, hv, sv = csr_arrays(H, S)
        a = lambda x: np.ascontiguousarray(x, dtype=np.int32)
        pe, cb, ss, se, ce = a(plend), a(cblk), a(surfstart), a(surfend), a(contend)
        did = ctypes.c_int32()
        self._check(self._L.negf_b200_upload_csr(
            self._h, rp.size - 1, int(ci.size), _i(rp), _i(ci), _d(hv.view(np.float64)),
            _d(sv.view(np.float64)) if sv is not None else None, pe.size, _i(pe), cb.size, _i(cb), _i(ss), _i(se),
            _i(ce), ctypes.byref(did)), "upload_csr")
        starts = np.concatenate([[0], pe[:-1]])
        self.devices[did.value] = DeviceShape(pl_size=[int(x) for x in pe - starts], cblk=[int(x) for x in cb],
                                              lead_size=[int(x) for x in (ce - ss + 1) // 2])
        return did.value

    def set_tun_proj(self, device_id, tun_proj):
        """tun_proj (1-based orbital indices) of the device; None or [] = whole trace."""
        idx = tun_indices(tun_proj if tun_proj is not None else [])
        self._check(self._L.negf_b200_set_tun_proj(self._h, device_id, idx.size, _i(idx) if idx.size else None),
                    "set_tun_proj")

    def set_dos_proj(self, device_id, dos_proj):
        """dos_proj (list of 1-based orbital index sets) of the device; None or [] = none."""
        if not dos_proj:
            self._check(self._L.negf_b200_set_dos_proj(self._h, device_id, 0, None, None), "set_dos_proj")
            self._nldos[device_id] = 0
            return
        ptr, idx = dos_sets(dos_proj)
        self._check(self._L.negf_b200_set_dos_proj(self._h, device_id, ptr.size - 1, _i(ptr), _i(idx)),
                    "set_dos_proj")
        self._nldos[device_id] = ptr.size - 1

    def transmissions(self, device_id, energies, pairs, eta=1e-4, ldos=False, dos_delta=1e-4, check=True):
        """T over contact pairs [(ni, nf), ...] (npts x npairs); with ldos=True
        also the LDOS of the device's dos_proj sets (npts x nsets)."""
        E = np.ascontiguousarray(energies, dtype=np.float64).ravel()
        n = E.size
        ids = self._ids(device_id, n)
        ni = np.ascontiguousarray([p[0] for p in pairs], dtype=np.int32)
        nf = np.ascontiguousarray([p[1] for p in pairs], dtype=np.int32)
        T = np.zeros((n, ni.size))
        nsets = max(self._nldos.get(int(i), 0) for i in set(ids.tolist())) if ldos else 0
        led = np.zeros((n, max(nsets, 1))) if ldos else None
        ncyc = np.zeros(n, dtype=np.int32)
        st = np.zeros(n, dtype=np.int32)
        rc = self._L.negf_b200_transmissions(self._h, n, _i(ids), _d(E), eta, dos_delta, ni.size, _i(ni), _i(nf),
                                             _d(T), _d(led) if ldos else None, _i(ncyc), _i(st))
        if (check or rc in CALL_ERRORS) and rc not in (OK, NOT_CONVERGED):
            raise NegfError(rc, "transmissions: " + self.last_error())
        return T, (led[:, :nsets] if ldos else None), ncyc, st

    def set_sgf_cache(self, mode: int, nbytes: int = 0):
        """Surface Green's function cache: 0 off, 1 reuse, 2 refresh."""
        self._check(self._L.negf_b200_set_sgf_cache(self._h, mode, nbytes), "set_sgf_cache")

    def set_workspace_limit(self, nbytes: int):
        """Caps the engine workspace (0 = none); see negf_b200_set_workspace_limit."""
        self._check(self._L.negf_b200_set_workspace_limit(self._h, nbytes), "set_workspace_limit")

    def sgf_cache_save(self, path) -> int:
        """Writes the cached surface GFs to `path`; returns the entry count."""
        n = ctypes.c_int64()
        self._check(self._L.negf_b200_sgf_cache_save(self._h, os.fsencode(path), ctypes.byref(n)), "sgf_cache_save")
        return n.value

    def sgf_cache_load(self, path) -> int:
        """Adds the entries of `path` for the uploaded devices' leads; returns
        the number of file entries used."""
        n = ctypes.c_int64()
        self._check(self._L.negf_b200_sgf_cache_load(self._h, os.fsencode(path), ctypes.byref(n)), "sgf_cache_load")
        return n.value

    def sgf_cache_stats(self) -> dict:
        h, m, e = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        b = ctypes.c_size_t()
        self._check(self._L.negf_b200_sgf_cache_stats(self._h, ctypes.byref(h), ctypes.byref(m), ctypes.byref(e),
                                                      ctypes.byref(b)), "sgf_cache_stats")
        return {"hits": h.value, "misses": m.value, "entries": e.value, "bytes": b.value}

    def density(self, device_id, z, w, pl=None, check=True):
        """Equilibrium density-matrix blocks from the contour points z with
        weights w (see negf_b200_density): (diag, upper, lower) block lists,
        the outer (device->contact, contact->device) blocks per contact,
        ncyc, status."""
        from .density import split_blocks, split_outer
        dev = self.devices[device_id]
        pl = pl if pl is not None else dev.pl_size
        nm = sum(dev.pl_size[cb - 1] * L for cb, L in zip(dev.cblk, dev.lead_size))
        rdc = np.zeros(max(nm, 1), dtype=np.complex128)
        rcd = np.zeros(max(nm, 1), dtype=np.complex128)
        z = np.ascontiguousarray(z, dtype=np.complex128).ravel()
        wt = np.ascontiguousarray(w, dtype=np.complex128).ravel()
        er, ei = np.ascontiguousarray(z.real), np.ascontiguousarray(z.imag)
        nd = sum(x * x for x in pl)
        no = sum(pl[i] * pl[i + 1] for i in range(len(pl) - 1))
        rd = np.zeros(max(nd, 1), dtype=np.complex128)
        ru = np.zeros(max(no, 1), dtype=np.complex128)
        rl = np.zeros(max(no, 1), dtype=np.complex128)
        nc = np.zeros(z.size, dtype=np.int32)
        st = np.zeros(z.size, dtype=np.int32)
        rc = self._L.negf_b200_density(self._h, device_id, z.size, _d(er), _d(ei), _d(wt.view(np.float64)),
                                       _d(rd.view(np.float64)), _d(ru.view(np.float64)), _d(rl.view(np.float64)),
                                       _d(rdc.view(np.float64)), _d(rcd.view(np.float64)), _i(nc), _i(st))
        if (check or rc in CALL_ERRORS) and rc not in (OK, NOT_CONVERGED):
            raise NegfError(rc, "density: " + self.last_error())
        return split_blocks(pl, rd, ru, rl), split_outer(dev, rdc, rcd), nc, st

    def density_neq(self, device_id, energies, w, frm, eta=1e-4, coupling=None, check=True):
        """Real-axis non-equilibrium density blocks sum_p w_p Gn(E_p) (see
        negf_b200_density_neq); frm: npts x ncont, reference contact
        subtracted.  Returns (diag, upper, lower) block lists, the outer
        (device->contact, contact->device) blocks per contact, ncyc, status."""
        from .density import split_blocks, split_outer
        dev = self.devices[device_id]
        pl = dev.pl_size
        nm = sum(dev.pl_size[cb - 1] * L for cb, L in zip(dev.cblk, dev.lead_size))
        rdc = np.zeros(max(nm, 1), dtype=np.complex128)
        rcd = np.zeros(max(nm, 1), dtype=np.complex128)
        E = np.ascontiguousarray(energies, dtype=np.float64).ravel()
        wt = np.ascontiguousarray(w, dtype=np.complex128).ravel()
        f = np.ascontiguousarray(frm, dtype=np.float64)
        cp = None if coupling is None else np.ascontiguousarray(coupling, dtype=np.float64)
        nd = sum(x * x for x in pl)
        no = sum(pl[i] * pl[i + 1] for i in range(len(pl) - 1))
        rd = np.zeros(max(nd, 1), dtype=np.complex128)
        ru = np.zeros(max(no, 1), dtype=np.complex128)
        rl = np.zeros(max(no, 1), dtype=np.complex128)
        nc = np.zeros(E.size, dtype=np.int32)
        st = np.zeros(E.size, dtype=np.int32)
        rc = self._L.negf_b200_density_neq(self._h, device_id, E.size, _d(E), eta, _d(wt.view(np.float64)), _d(f),
                                           _d(cp) if cp is not None else None, _d(rd.view(np.float64)),
                                           _d(ru.view(np.float64)), _d(rl.view(np.float64)),
                                           _d(rdc.view(np.float64)), _d(rcd.view(np.float64)), _i(nc), _i(st))
        if (check or rc in CALL_ERRORS) and rc not in (OK, NOT_CONVERGED, SCBA_NOT_CONVERGED):
            raise NegfError(rc, "density_neq: " + self.last_error())
        return split_blocks(pl, rd, ru, rl), split_outer(dev, rdc, rcd), nc, st

    def release(self, device_id: int):
        self._check(self._L.negf_b200_release_device(self._h, device_id), "release")
        self.devices.pop(device_id, None)

    # -- solves (host buffers)
    @staticmethod
    def _ids(device_id, npts):
        return np.ascontiguousarray(np.broadcast_to(np.asarray(device_id, dtype=np.int32), (npts,)))

    def transmission(self, device_id, energies, eta=1e-4, ni=1, nf=2, check=True):
        E = np.ascontiguousarray(energies, dtype=np.float64).ravel()
        n = E.size
        ids = self._ids(device_id, n)
        T = np.zeros(n)
        ncyc = np.zeros(n, dtype=np.int32)
        st = np.zeros(n, dtype=np.int32)
        rc = self._L.negf_b200_transmission(self._h, n, _i(ids), _d(E), eta, ni, nf, _d(T), _i(ncyc), _i(st))
        if (check or rc in CALL_ERRORS) and rc not in (OK, NOT_CONVERGED):
            raise NegfError(rc, "transmission: " + self.last_error())
        return T, ncyc, st

    def transmission_dos(self, device_id, energies, eta=1e-4, dos_delta=1e-4, ni=1, nf=2, check=True):
        E = np.ascontiguousarray(energies, dtype=np.float64).ravel()
        n = E.size
        ids = self._ids(device_id, n)
        norb = max(self.devices[int(i)].norb for i in set(ids.tolist()))
        T = np.zeros(n)
        dos = np.zeros((n, norb))
        ncyc = np.zeros(n, dtype=np.int32)
        st = np.zeros(n, dtype=np.int32)
        rc = self._L.negf_b200_transmission_dos(self._h, n, _i(ids), _d(E), eta, dos_delta, ni, nf, _d(T), _d(dos),
                                                _i(ncyc), _i(st))
        if (check or rc in CALL_ERRORS) and rc not in (OK, NOT_CONVERGED):
            raise NegfError(rc, "transmission_dos: " + self.last_error())
        return T, dos, ncyc, st

    def meir_wingreen(self, device_id, energies, frm, coupling=None, eta=1e-4, check=True):
        E = np.ascontiguousarray(energies, dtype=np.float64).ravel()
        n = E.size
        ids = self._ids(device_id, n)
        devs = [self.devices[int(i)] for i in set(ids.tolist())]
        ncont = max(d.ncont for d in devs)
        nbl = max(d.nbl for d in devs)
        norb = max(d.norb for d in devs)
        frm = np.ascontiguousarray(np.broadcast_to(np.asarray(frm, dtype=np.float64), (n, ncont)))
        cp = None if coupling is None else np.ascontiguousarray(
            np.broadcast_to(np.asarray(coupling, dtype=np.float64), (norb,)))
        curr = np.zeros((n, ncont))
        lcurr = np.zeros((n, max(nbl - 1, 1)))
        ldens = np.zeros((n, nbl))
        it = np.zeros(n, dtype=np.int32)
        err = np.zeros(n)
        ncyc = np.zeros(n, dtype=np.int32)
        st = np.zeros(n, dtype=np.int32)
        rc = self._L.negf_b200_meir_wingreen(self._h, n, _i(ids), _d(E), eta, _d(frm), _d(cp), _d(curr), _d(lcurr),
                                             _d(ldens), _i(it), _d(err), _i(ncyc), _i(st))
        if (check or rc in CALL_ERRORS) and rc not in (OK, NOT_CONVERGED):
            raise NegfError(rc, "meir_wingreen: " + self.last_error())
        return dict(curr=curr, layer_curr=lcurr[:, :nbl - 1], layer_dens=ldens, scba_iter=it, scba_err=err,
                    ncyc=ncyc, status=st)


def version() -> str:
    return load().negf_b200_version().decode()
