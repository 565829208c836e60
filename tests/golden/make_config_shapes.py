"""Writes tests/golden/config_shapes.npz: parity fixtures at the shapes of
the four solve workloads, on the seeded generators' devices.

  c0  20 layers x 32 orbitals, S = I, all 512 energies of [-3, 3] eV,
      eta = 1e-6, surface Green's functions converged to SGFACC = 1e-12;
      T(E).
  c1  100 layers x 256 orbitals, S = I + 0.05 R, 8 points over two
      transverse k-points, eta = 1e-6, SGFACC = 1e-9; T(E,k) and the
      diagonal spectral density (every 16th orbital stored).
  c2  60 layers x 512 orbitals (the c1 generator), 4 grid energies over two
      k-points and 4 energies within 1e-3 eV of a lead band edge, eta =
      1e-6, SGFACC = 1e-9; T(E,k).
  c3  40 layers x 128 orbitals (the c0 generator), elastic dephasing with
      coupling 0.1 eV on every orbital, 0.2 eV bias, 300 K, linear mixing
      0.5 until the contact-1 current changes by < 1e-8 (at most 100
      sweeps); contact currents, layer currents and densities, sweep counts.

For the T and T + DOS shapes four CPU solutions are stored per point:
  T_o   the oracle (LAPACK zgetrf/zgetrs + zgemm, the reference's sequence);
  T_d   the same algorithm in double with its own unblocked LU and
        triple-loop products (a second FP64 rounding path);
  T_g   the same in double with Gauss-Jordan inverses (a third one, with the
        elimination order of the engine's inversion);
  T_x   the same algorithm in long double (64-bit significand), a near-exact
        solution: |T_o - T_x| is the reference path's own rounding error;
  T_s   the oracle's largest change under two rounding-level (1e-15
        relative) perturbations of every input block.
At energies where the device solve is ill-conditioned (the device blocks
carry no broadening, src/integrations.F90:1747-1752, so narrow resonances
are only as wide as the lead coupling makes them) the FP64 paths land up to
1e-7 relative away from T_x; the parity tests list the points where any of
them lands beyond an eighth of the 1e-10 bound.

Each device is generated again by the tests from its seed; the stored
fingerprint (sha256 of every block) makes a changed generator fail loudly.

Run:  python tests/golden/make_config_shapes.py [c0 c1 c2 c3] [--kinds o,d,g,x]
      (c2's long-double solves take about forty minutes on eight cores;
      --kinds recomputes only the named solutions and keeps the others)
"""
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from libnegf_b200 import generators as G   # noqa: E402

PATH = os.path.join(HERE, "config_shapes.npz")
BLOCK_LISTS = ("h_diag", "h_upper", "h_lower", "s_diag", "s_upper", "s_lower",
               "lead_h00", "lead_h01", "lead_s00", "lead_s01", "hmc", "smc")
DOS_STRIDE = 16


def fingerprint(dev):
    h = hashlib.sha256()
    h.update(np.asarray(dev.cblk, dtype=np.int64).tobytes())
    for k in BLOCK_LISTS:
        lst = getattr(dev, k)
        if lst is None:
            continue
        for b in lst:
            h.update(np.ascontiguousarray(b, dtype=np.complex128).tobytes())
    return h.hexdigest()


# ------------------------------------------------------------------ shapes
def c0_case():
    dev = G.transport_c0(nbl=20, n=32, seed=0)
    E = G.energy_grid(-3.0, 3.0, 512)
    return [dev], np.zeros(E.size, dtype=np.int32), E, dict(eta=1e-6, sgf_tol=1e-12, dos=False)


C1_K = (0, 5)     # of the 16 transverse k-points pi*j/16


def c1_case():
    ks = [np.pi * j / 16 for j in C1_K]
    devs = G.transport_c1_kpoints(ks, nbl=100, n=256, seed=1)
    grid = G.energy_grid(-2.0, 2.0, 2048)
    sel = np.array([150, 700, 1300, 1900])
    ids = np.repeat(np.arange(len(ks), dtype=np.int32), sel.size)
    E = np.concatenate([grid[sel], grid[sel + 37]])
    return devs, ids, E, dict(eta=1e-6, sgf_tol=1e-9, dos=True)


C2_K = (0, 3)     # of the 8 transverse k-points pi*j/8


def c2_case():
    ks = [np.pi * j / 8 for j in C2_K]
    devs = G.transport_c1_kpoints(ks, nbl=60, n=512, seed=1)
    grid = G.energy_grid(-2.0, 2.0, 1024)
    edge = G.band_edge_energies(devs[0], contact=0, nk=64, n_edges=64, window=1e-3)
    edge = edge[np.linspace(0, edge.size - 1, 4).astype(int)]
    ids = np.array([0, 0, 1, 1, 0, 0, 0, 0], dtype=np.int32)
    E = np.concatenate([grid[[200, 800]], grid[[333, 640]], edge])
    return devs, ids, E, dict(eta=1e-6, sgf_tol=1e-9, dos=False)


C3_SCBA = dict(coupling=0.1, bias=0.2, temp_k=300.0, niter=100, tol=1e-8, mix=0.5, rule=1, eta=1e-4)


def c3_case():
    dev = G.transport_c0(nbl=40, n=128, seed=0)
    grid = G.energy_grid(-1.0, 1.0, 1024)
    E = grid[[100, 480, 530, 900]]
    return [dev], np.zeros(E.size, dtype=np.int32), E, dict(C3_SCBA)


def c3_occupations(E):
    """Contact occupations f_c = fermi(E, mu_c, kT) at mu = +-bias/2, the
    reference occupation 0 (src/integrations.F90:1883-1887)."""
    from libnegf_b200.energy import fermi_f
    kt = 8.617333262e-5 * C3_SCBA["temp_k"]
    mu = (0.5 * C3_SCBA["bias"], -0.5 * C3_SCBA["bias"])
    return np.ascontiguousarray(np.stack([fermi_f(E, mu[0], kt), fermi_f(E, mu[1], kt)], axis=1))


CASES = {"c0": c0_case, "c1": c1_case, "c2": c2_case, "c3": c3_case}


KINDS = ("o", "d", "g", "x", "s")


def perturbed(dev, rng, rel=1e-15):
    """Copy of `dev` with every block element scaled by (1 + rel N(0,1))."""
    import copy
    d = copy.deepcopy(dev)
    for name in BLOCK_LISTS:
        lst = getattr(d, name)
        if lst is None:
            continue
        for i in range(len(lst)):
            lst[i] = lst[i] * (1.0 + rel * rng.standard_normal(lst[i].shape))
    return d


def run_shape(name, out, kinds=KINDS):
    from oracle import oracle as O
    devs, ids, E, p = CASES[name]()
    for k, d in enumerate(devs):
        out["%s__fp%d" % (name, k)] = np.array(fingerprint(d))
    out[name + "__ids"] = ids
    out[name + "__E"] = E
    if name == "c3":
        frm = c3_occupations(E)
        cpl = np.full(devs[0].norb, C3_SCBA["coupling"])
        r = O.meir_wingreen(devs[0], E, frm, coupling=cpl, eta=p["eta"], scba_niter=p["niter"],
                            scba_tol=p["tol"], scba_mix=p["mix"], scba_rule=p["rule"])
        for k in ("curr", "layer_curr", "layer_dens", "scba_iter", "ncyc", "status"):
            out["c3__o_" + k] = np.asarray(r[k])
        return
    n = E.size
    for key in kinds:
        T = np.zeros(n)
        nc = np.zeros(n, dtype=np.int32)
        dos = None
        for k, d in enumerate(devs):
            sel = np.nonzero(ids == k)[0]
            if sel.size == 0:
                continue
            Ek = E[sel]
            t0 = time.time()
            if key == "s":
                rng = np.random.default_rng(17)
                t = np.zeros(sel.size)
                ds = None
                base = (O.transmission_dos(d, Ek, eta=p["eta"], dos_delta=0.0, sgf_tol=p["sgf_tol"]) if p["dos"]
                        else O.transmission(d, Ek, eta=p["eta"], sgf_tol=p["sgf_tol"]))
                for _ in range(2):
                    dp = perturbed(d, rng)
                    r = (O.transmission_dos(dp, Ek, eta=p["eta"], dos_delta=0.0, sgf_tol=p["sgf_tol"]) if p["dos"]
                         else O.transmission(dp, Ek, eta=p["eta"], sgf_tol=p["sgf_tol"]))
                    t = np.maximum(t, np.abs(r[0] - base[0]))
                    if p["dos"]:
                        dd = np.abs(r[1] - base[1])
                        ds = dd if ds is None else np.maximum(ds, dd)
                c, st = base[-2], base[-1]
            elif key == "o" and p["dos"]:
                t, ds, c, st = O.transmission_dos(d, Ek, eta=p["eta"], dos_delta=0.0, sgf_tol=p["sgf_tol"])
            elif key == "o":
                t, c, st = O.transmission(d, Ek, eta=p["eta"], sgf_tol=p["sgf_tol"])
                ds = None
            else:
                t, ds, c, st = O.transmission_xp(d, Ek, eta=p["eta"], dos_delta=0.0 if p["dos"] else None,
                                                 sgf_tol=p["sgf_tol"], extended=(key == "x"),
                                                 gauss_jordan=(key == "g"))
            print("  %s k=%d %s: %d points in %.1f s" % (name, k, key, sel.size, time.time() - t0), flush=True)
            assert np.all(st == 0), st
            T[sel], nc[sel] = t, c
            if ds is not None:
                dos = dos if dos is not None else np.zeros((n, ds.shape[1]))
                dos[sel] = ds
        out["%s__T_%s" % (name, key)] = T
        out["%s__ncyc_%s" % (name, key)] = nc
        if dos is not None:
            out["%s__dos_%s" % (name, key)] = dos[:, ::DOS_STRIDE].copy()


def main(names, kinds=KINDS):
    out = {}
    if os.path.exists(PATH):
        z = np.load(PATH)
        out = {k: z[k] for k in z.files}
    for name in names:
        if set(kinds) == set(KINDS) or name == "c3":
            for k in [k for k in out if k.startswith(name + "__")]:
                del out[k]
        t0 = time.time()
        run_shape(name, out, kinds)
        print("%s done in %.1f s" % (name, time.time() - t0), flush=True)
        np.savez_compressed(PATH, **out)
    print("wrote", PATH)


if __name__ == "__main__":
    args = sys.argv[1:]
    kinds = KINDS
    if "--kinds" in args:
        i = args.index("--kinds")
        kinds = tuple(args[i + 1].split(","))
        del args[i:i + 2]
    main(args or list(CASES), kinds)
