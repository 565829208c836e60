"""Committed golden fixtures (tests/golden/golden.npz, written by
tests/golden/make_golden.py): the oracle must still reproduce them (CPU), and
the CUDA path must match them through the C-ABI (GPU).

Bounds, as in the other parity tests: T 1e-10 relative / 1e-13 absolute;
DOS, LDOS, currents, densities and density-matrix blocks 1e-10 relative to
the largest entry; each widened to 10x the oracle's own spread under
rounding-level input perturbations (the eta = 1e-6 solve and the sharp
DOS peaks at dos_delta = 1e-4 amplify rounding)."""
import os

import numpy as np
import pytest

from conftest import assert_T_close, oracle_spread, perturbed
from golden.make_golden import cases, load_device, run_case

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz")
PARAMS = {name: p for name, _, p in cases()}
NAMES = list(PARAMS)


@pytest.fixture(scope="module")
def golden():
    return np.load(PATH)


def outputs(z, name):
    pre = name + "__out__"
    return {k[len(pre):]: z[k] for k in z.files if k.startswith(pre)}


def _close_rel(a, b, rel=1e-10, spread=None):
    a, b = np.asarray(a), np.asarray(b)
    bound = rel * max(1.0, np.abs(b).max())
    if spread is not None:
        bound = np.maximum(bound, 10.0 * np.asarray(spread))
    return np.all(np.abs(a - b) <= bound)


def _check(name, got, ref, spread=None):
    sp = spread if isinstance(spread, dict) else {}
    for k, v in ref.items():
        if k in ("z", "w"):
            continue
        if k == "ncyc":
            assert np.all(np.abs(np.asarray(got[k]) - v) <= 1), "%s: ncyc" % name
        elif k == "scba_iter":
            assert np.all(np.abs(np.asarray(got[k]) - v) <= 1), "%s: scba_iter" % name
        elif k == "status":
            assert np.array_equal(np.asarray(got[k]), v), "%s: status" % name
        elif k == "T":
            assert_T_close(got[k], v, what="%s %s" % (name, k), spread=sp.get(k))
        else:
            assert _close_rel(got[k], v, spread=sp.get(k)), "%s: %s" % (name, k)


def test_fixture_devices_load(golden):
    for name in NAMES:
        dev = load_device(golden, name)
        dev.validate()
        assert dev.norb > 0


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden(golden, name):
    dev = load_device(golden, name)
    got = run_case(dev, PARAMS[name])
    ref = outputs(golden, name)
    assert set(got) == set(ref)
    if PARAMS[name].get("eta", 1e-4) < 1e-5:
        _, spread = oracle_spread(lambda d: run_case(d, PARAMS[name])["T"], dev)
        _check(name, got, ref, {"T": spread})
    else:
        _check(name, got, ref)


def _spread(dev, p, nsamp=3):
    """The oracle's own change (complex modulus for complex outputs) under
    rounding-level perturbations of the device blocks."""
    rng = np.random.default_rng(0)
    ref = run_case(dev, p)
    out = {k: np.zeros(np.shape(v)) for k, v in ref.items()}
    for _ in range(nsamp):
        r = run_case(perturbed(dev, rng), p)
        for k in out:
            out[k] = np.maximum(out[k], np.abs(np.asarray(r[k]) - np.asarray(ref[k])))
    return out


def _gpu_run(ctx, dev, p):
    """The same quantities as run_case, computed by the CUDA path."""
    did = ctx.upload(dev)
    try:
        if p["kind"] == "tdos":
            T, dos, nc, st = ctx.transmission_dos(did, p["E"], eta=p["eta"], dos_delta=p["dos_delta"])
            return dict(T=T, dos=dos, ncyc=nc, status=st)
        if p["kind"] == "t":
            T, nc, st = ctx.transmission(did, p["E"], eta=p["eta"])
            return dict(T=T, ncyc=nc, status=st)
        if p["kind"] == "pairs":
            ctx.set_dos_proj(did, p["dos_proj"])
            T, led, nc, st = ctx.transmissions(did, p["E"], p["pairs"], eta=p["eta"], ldos=True,
                                               dos_delta=p["dos_delta"])
            return dict(T=T, ledos=led, ncyc=nc, status=st)
        if p["kind"] == "scba":
            ctx.set_options(scba_niter=p["niter"])
            try:
                r = ctx.meir_wingreen(did, p["E"], p["frm"], coupling=np.full(dev.norb, p["coupling"]), eta=p["eta"])
            finally:
                ctx.set_options()
            return dict(curr=r["curr"], layer_curr=r["layer_curr"], layer_dens=r["layer_dens"],
                        scba_iter=r["scba_iter"], ncyc=r["ncyc"], status=r["status"])
        if p["kind"] == "rho":
            raise AssertionError("rho runs from the stored contour points")
    finally:
        ctx.release(did)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_matches_golden(gpu_ctx, golden, name):
    dev = load_device(golden, name)
    p = PARAMS[name]
    ref = outputs(golden, name)
    if p["kind"] == "rho":
        did = gpu_ctx.upload(dev)
        try:
            (d, u, l), _, nc, st = gpu_ctx.density(did, ref["z"], ref["w"])
        finally:
            gpu_ctx.release(did)
        got = dict(rho_diag=np.stack(d), rho_upper=np.stack(u), rho_lower=np.stack(l), ncyc=nc, status=st)
    else:
        got = _gpu_run(gpu_ctx, dev, p)
    _check(name, got, ref, _spread(dev, p))
