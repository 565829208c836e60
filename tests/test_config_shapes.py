"""GPU parity at the shapes of the solve workloads (tests/golden/config_shapes.npz,
written by tests/golden/make_config_shapes.py):

  c0  20 x 32, all 512 energies, eta = 1e-6, SGFACC = 1e-12, T(E);
  c1  100 x 256, S = I + 0.05 R, 8 points over two k-points, T + DOS;
  c2  60 x 512, 4 grid energies and 4 energies within 1e-3 eV of a lead
      band edge, T;
  c3  40 x 128 elastic-dephasing SCBA (mixing 0.5, current-change rule).

The bound is the north star's: 1e-10 relative where T > 1e-6 and 1e-13
absolute otherwise, strict at every point where three CPU FP64 paths of the
same algorithm (the oracle's LAPACK one, an unblocked LU one, a Gauss-Jordan
one) all lie within an eighth of it from the long-double solution, and so
does the oracle's own change under rounding-level input perturbations.  The
remaining points are listed by that measurement (the fixture holds all CPU
solutions and the spread); there the GPU result must be as close to the
long-double solution as the CPU FP64 paths are.  The decimation's iteration
count equals the oracle's at every point."""
import numpy as np
import pytest

from conftest import assert_parity, assert_T_strict
from golden.make_config_shapes import C3_SCBA, CASES, DOS_STRIDE, PATH, c3_occupations, fingerprint

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fixture():
    return np.load(PATH)


def _upload(ctx, z, shape):
    """The fixture's devices (regenerated, checked bit for bit) and energies
    (taken from the fixture: band-edge energies come from an eigensolver
    whose last bits depend on the host CPU)."""
    devs, ids, E, p = CASES[shape]()
    for k, d in enumerate(devs):
        assert fingerprint(d) == str(z["%s__fp%d" % (shape, k)]), "generator changed: regenerate the fixture"
    assert np.array_equal(ids, z[shape + "__ids"]) and np.allclose(E, z[shape + "__E"], rtol=1e-12, atol=0)
    E = np.array(z[shape + "__E"])
    handles = [ctx.upload(d) for d in devs]
    return devs, np.asarray(handles, dtype=np.int32)[ids], E, p, handles


@pytest.mark.parametrize("shape", ["c0", "c1", "c2"])
def test_config_shape_transmission(gpu_ctx, fixture, shape):
    z = fixture
    devs, hid, E, p, handles = _upload(gpu_ctx, z, shape)
    gpu_ctx.set_options(sgf_tol=p["sgf_tol"])
    try:
        if p["dos"]:
            T, dos, ncyc, st = gpu_ctx.transmission_dos(hid, E, eta=p["eta"], dos_delta=0.0)
        else:
            T, ncyc, st = gpu_ctx.transmission(hid, E, eta=p["eta"])
            dos = None
        assert np.all(st == 0)
        assert np.array_equal(ncyc, z[shape + "__ncyc_o"]), "decimation iteration counts differ from the oracle"
        x = {"T_x": z[shape + "__T_x"], "T_d": z[shape + "__T_d"], "T_g": z[shape + "__T_g"]}
        listed = assert_T_strict(T, z[shape + "__T_o"], x, spread=z[shape + "__T_s"], what=shape + " T")
        print("%s: %d points, %d listed (CPU FP64 paths beyond an eighth of the bound from long double): E = %s" % (
            shape, E.size, listed.size, np.array2string(E[listed], precision=5)))
        if dos is not None:
            ref = z[shape + "__dos_o"]
            bound = 1e-10 * max(np.abs(ref).max(), 1.0)
            assert_parity(dos[:, ::DOS_STRIDE], ref, bound, ref_x=z[shape + "__dos_x"],
                          others=(z[shape + "__dos_d"], z[shape + "__dos_g"]), spread=z[shape + "__dos_s"],
                          what=shape + " DOS", rows=True)
    finally:
        gpu_ctx.set_options()
        for h in handles:
            gpu_ctx.release(h)


def test_config_shape_scba(gpu_ctx, fixture):
    z = fixture
    devs, hid, E, p, handles = _upload(gpu_ctx, z, "c3")
    gpu_ctx.set_options(scba_niter=C3_SCBA["niter"], scba_tol=C3_SCBA["tol"], scba_mix=C3_SCBA["mix"],
                        scba_rule=C3_SCBA["rule"])
    try:
        cpl = np.full(devs[0].norb, C3_SCBA["coupling"])
        r = gpu_ctx.meir_wingreen(hid, E, c3_occupations(E), coupling=cpl, eta=C3_SCBA["eta"], check=False)
        assert np.array_equal(r["status"], z["c3__o_status"])
        assert np.array_equal(r["ncyc"], z["c3__o_ncyc"])
        assert np.array_equal(r["scba_iter"], z["c3__o_scba_iter"])
        for key in ("curr", "layer_curr", "layer_dens"):
            ref = z["c3__o_" + key]
            err = np.abs(r[key] - ref).max()
            assert err <= 1e-10 * max(1.0, np.abs(ref).max()), (key, err)
    finally:
        gpu_ctx.set_options()
        for h in handles:
            gpu_ctx.release(h)
