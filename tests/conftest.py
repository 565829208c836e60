import copy
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def perturbed(dev, rng, rel=1e-15):
    """Copy of `dev` with every H/S/contact block element scaled by
    (1 + rel*N(0,1)): a rounding-level change of the inputs."""
    d = copy.deepcopy(dev)
    for name in ("h_diag", "h_upper", "h_lower", "s_diag", "s_upper", "s_lower",
                 "lead_h00", "lead_h01", "lead_s00", "lead_s01", "hmc", "smc"):
        lst = getattr(d, name)
        if lst is None:
            continue
        for i in range(len(lst)):
            lst[i] = lst[i] * (1.0 + rel * rng.standard_normal(lst[i].shape))
    return d


def oracle_spread(run, dev, nsamp=3, seed=0):
    """Reference output and its own reproducibility: the largest change of
    run(dev) (an array or a dict of arrays) over `nsamp` rounding-level
    perturbations of the inputs."""
    rng = np.random.default_rng(seed)
    ref = run(dev)
    keys = list(ref) if isinstance(ref, dict) else [None]
    get = (lambda r, k: np.asarray(r[k], dtype=float)) if keys[0] is not None else (lambda r, k: np.asarray(r, float))
    spread = {k: np.zeros_like(get(ref, k)) for k in keys}
    for _ in range(nsamp):
        r = run(perturbed(dev, rng))
        for k in keys:
            spread[k] = np.maximum(spread[k], np.abs(get(r, k) - get(ref, k)))
    return ref, (spread if keys[0] is not None else spread[None])


def assert_T_close(T, Tref, rtol=1e-10, atol=1e-13, what="T", spread=None, kspread=10.0):
    """Transmission parity bound: |T - Tref| <= max(rtol*|Tref|, atol).

    This is the 1e-10 relative / 1e-13 absolute bound, with the absolute
    floor applied everywhere: the reference's 2-contact formula
    T = |Re Tr[Gam A] - Re Tr[Gam G Gam G^dag]| (iterative_cpu.F90:438-464)
    subtracts two traces of order Tr[Gam A] ~ 1, so any two correct
    implementations (two LAPACK builds included) differ by ~1e-14 absolute
    even where T is only slightly above 1e-6.

    `spread` (optional, per point): the oracle's own change under
    rounding-level (1e-15 relative) perturbations of the inputs.  With
    eta = 1e-6 the decimation amplifies rounding by up to ~1e6 near lead band
    edges, so there the bound is kspread * spread instead of 1e-10."""
    T = np.asarray(T, dtype=float)
    Tref = np.asarray(Tref, dtype=float)
    assert T.shape == Tref.shape
    err = np.abs(T - Tref)
    bound = np.maximum(rtol * np.abs(Tref), atol)
    if spread is not None:
        # the oracle's own reproducibility under rounding-level input changes
        bound = np.maximum(bound, kspread * np.asarray(spread, dtype=float))
    bad = err > bound
    assert not bad.any(), "%s: %d points out of bound; worst err %.3e at Tref=%.3e" % (
        what, int(bad.sum()), err[bad].max(), Tref[bad][np.argmax(err[bad])])


def xp_reference(dev, E, eta, dos_delta=None, sgf_tol=1e-9):
    """The long-double solution of the oracle's 2-contact T (or T + DOS) path
    and two more FP64 rounding paths of the same algorithm (own unblocked LU
    and products; Gauss-Jordan inverses), or None where that restatement does
    not cover the device (not 2 contacts, or a T-only solve off the fast
    path)."""
    from oracle import oracle as O
    if dev.ncont != 2 or (dos_delta is None and min(dev.cblk) != 1):
        return None
    kw = dict(eta=eta, dos_delta=dos_delta, sgf_tol=sgf_tol)
    x = O.transmission_xp(dev, E, extended=True, **kw)
    d = O.transmission_xp(dev, E, extended=False, **kw)
    g = O.transmission_xp(dev, E, extended=False, gauss_jordan=True, **kw)
    return {"T_x": x[0], "dos_x": x[1], "ncyc_x": x[2], "T_d": d[0], "dos_d": d[1], "T_g": g[0], "dos_g": g[1]}


LIST_FRACTION = 0.125


def fp64_scatter(ref, ref_x, others=()):
    """Largest distance of the FP64 results (the oracle's and the other CPU
    rounding paths') from the long-double solution, per point."""
    e = np.abs(np.asarray(ref, dtype=float) - ref_x)
    for o in others:
        if o is not None:
            e = np.maximum(e, np.abs(np.asarray(o, dtype=float) - ref_x))
    return e


def assert_parity(got, ref, bound, ref_x=None, others=(), spread=None, what="T", kx=10.0, rows=False):
    """Parity of `got` against the oracle `ref` at the bound (an array).

    The FP64 rounding of the reference path is sampled per point by the CPU
    FP64 paths' distances from the long-double solution `ref_x` (the
    oracle's and the restated ones in `others`) and by `spread`, the
    oracle's own change under rounding-level (1e-15 relative) input
    perturbations.  Strict, |got - ref| <= bound, wherever every sample is
    within an eighth of the bound.  The other points are listed (returned,
    and named in a failure message): there the reference path's own FP64
    result scatters beyond the bound's margin, and the result must be as
    close to the long-double solution as the CPU FP64 paths are,
    |got - ref_x| <= max(bound, kx * the largest sample), or, without a
    long-double solution, |got - ref| <= max(bound, kx * spread).

    rows=True (a vector per point, e.g. the per-orbital DOS: points x
    entries): the listed entries of a point are held to kx times the largest
    sample over that point's entries.  A rounding-level change moves the
    whole vector of a point at once, in a direction that differs from sample
    to sample, so a handful of samples measures the point's scatter, not
    each entry's."""
    got = np.asarray(got, dtype=float)
    ref = np.asarray(ref, dtype=float)
    bound = np.broadcast_to(np.asarray(bound, dtype=float), ref.shape)
    assert got.shape == ref.shape
    e_cpu = np.zeros(ref.shape)
    if ref_x is not None:
        ref_x = np.asarray(ref_x, dtype=float)
        e_cpu = fp64_scatter(ref, ref_x, others)
    if spread is not None:
        e_cpu = np.maximum(e_cpu, np.asarray(spread, dtype=float))
    listed = e_cpu > LIST_FRACTION * bound
    err = np.abs(got - ref)
    bad = (~listed) & (err > bound)
    assert not bad.any(), "%s: %d of %d points beyond the strict bound; worst err %.3e (bound %.3e) at ref=%.6e" % (
        what, int(bad.sum()), bad.size, err[bad].max(), bound[bad][np.argmax(err[bad])],
        ref[bad][np.argmax(err[bad])])
    if listed.any():
        e_x = np.abs(got - (ref_x if ref_x is not None else ref))
        scale = np.broadcast_to(e_cpu.max(axis=1, keepdims=True), e_cpu.shape) if rows else e_cpu
        lim = np.maximum(bound, kx * scale)
        badx = listed & (e_x > lim)
        assert not badx.any(), (
            "%s: %d listed points farther from the %s than %gx the FP64 rounding samples: "
            "worst %.3e against %.3e" % (what, int(badx.sum()),
                                         "long-double solution" if ref_x is not None else "oracle",
                                         kx, e_x[badx].max(), scale[badx][np.argmax(e_x[badx])]))
    return np.nonzero(listed.ravel())[0]


def assert_T_strict(T, Tref, xref=None, spread=None, rtol=1e-10, atol=1e-13, what="T"):
    """The transmission bound |T - Tref| <= max(rtol |Tref|, atol), strict
    except at the points where the reference path's FP64 rounding scatters
    beyond an eighth of it (`xref` from xp_reference or the fixture, `spread`
    from oracle_spread)."""
    Tref = np.asarray(Tref, dtype=float)
    bound = np.maximum(rtol * np.abs(Tref), atol)
    if xref is None:
        return assert_parity(T, Tref, bound, spread=spread, what=what)
    return assert_parity(T, Tref, bound, ref_x=xref["T_x"], others=(xref["T_d"], xref.get("T_g")), spread=spread,
                         what=what)


@pytest.fixture(scope="session")
def gpu_ctx():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from libnegf_b200 import native
    ctx = native.Context(0)
    yield ctx
    ctx.close()
