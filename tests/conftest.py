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


@pytest.fixture(scope="session")
def gpu_ctx():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from libnegf_b200 import native
    ctx = native.Context(0)
    yield ctx
    ctx.close()
