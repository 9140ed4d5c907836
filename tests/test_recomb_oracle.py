"""The recombination-ray oracle (oracle/recomb.py) against the reference's
own code, and the golden fixture tests/golden/recomb16.npz (made by
tests/golden/make_golden_recomb.py from the reference) against the oracle:

- the LTE spectrum tables and draws: lte_fill() / lte_gen_freq()
  src/lte.c:36-72, read back from the reference build;
- the isothermal closed form with the recombination photons against a
  tight implicit integration of solve.c:83-86 (case A), and against the
  reference's LSODA to its tolerance;
- the fixture's recombination rays are the oracle's emission from the
  fixture's states; the emitters are the previous tick's marked particles;
  the photons leave the emitters' yGrecHII.
"""
import math

import numpy as np
import pytest

from conftest import load_golden

RTOL_LSODA_ABS = 3e-5     # LSODA (rtol 1e-4, atol 1e-7) on yGrecHII over one step


def _consts(phys):
    return {k: phys.unit(k) for k in ("HI_ENERGY", "BOLTZMANN", "H_PER_MASS", "MPROTON_OVER_BOLTZMANN", "hmf", "hemf")}


@pytest.fixture(scope="module")
def phys_rec(units, built):
    from psphray_b200 import api
    return api.Physics(units, isothermal=True, on_the_spot=False)


@pytest.fixture(scope="module")
def lte(phys_rec):
    import recomb
    c = _consts(phys_rec)
    return recomb.lte_table(c["HI_ENERGY"], c["BOLTZMANN"], lambda e: phys_rec.xs_get("HI", e), weights=True)


@pytest.mark.parametrize("species", [0, 1, 2])
def test_lte_tables_vs_reference(reference, phys_rec, species):
    """lte_fill() of the three species (HI, HeI, HeII recombinations)."""
    import recomb
    reference.lte_init()
    c = _consts(phys_rec)
    th = [c["HI_ENERGY"], phys_rec.unit("HEI_ENERGY"), phys_rec.unit("HEII_ENERGY")][species]
    sp = ("HI", "HeI", "HeII")[species]
    freq, cdf, wt = recomb.lte_table(th, c["BOLTZMANN"], lambda e: phys_rec.xs_get(sp, e), weights=True)
    for row in range(recomb.NLOGT):
        f, w = reference.lte_row(row, species)
        assert np.max(np.abs(f - freq) / freq) < 1e-15
        assert np.array_equal(w > 0, wt[row] > 0)
        big = w > 1e-290
        assert np.max(np.abs(wt[row][big] - w[big]) / w[big]) < 1e-11
    fstep = (16.0 * th - th) / recomb.NFREQ
    rng = np.random.default_rng(2 + species)
    for _ in range(1000):
        logT, u = rng.uniform(2.5, 10.5), rng.uniform()
        row = min(max(int((logT - 3.0) / (7.0 / recomb.NLOGT)), 0), recomb.NLOGT - 1)
        mine = th + fstep * recomb.lte_index(cdf[row], u)
        assert abs(mine - reference.lte_gen_freq(logT, u, species)) <= 1e-12 * mine


def test_iso_closed_form_vs_implicit(phys_rec):
    from scipy.integrate import solve_ivp
    import recomb
    g = load_golden("recomb16.npz")
    he_e = phys_rec.unit("hemf") / phys_rec.unit("hmf") * 0.5
    for i in range(0, len(g["iso_in_lambdaH"]), 4):
        lam0, gd, tm, nH, T = (float(g[f"iso_in_{k}"][i]) for k in ("lambdaH", "yGdepHI", "time", "nH", "T"))
        lam1, dy = recomb.iso_step(lam0, gd, tm, nH, T, 0.0, he_e, phys_rec.ar_get)
        lt = math.log10(T)
        gam, aA, aB = (phys_rec.ar_get(k, lt) * nH for k in ("HIci", "HIIrcA", "HIIrcB"))
        aab = max(aA - aB, 0.0)

        def f(s, x):
            ye = 1.0 - x[0] + he_e
            return [-gd + tm * ye * (aA * (1 - x[0]) - gam * x[0]), tm * aab * ye * (1 - x[0])]
        sol = solve_ivp(f, (0, 1), [lam0, 0.0], method="Radau", rtol=1e-12, atol=1e-15)
        assert abs(lam1 - sol.y[0, -1]) < 1e-9
        assert abs(dy - sol.y[1, -1]) <= 1e-9 * abs(sol.y[1, -1]) + 1e-15


def test_iso_closed_form_vs_lsoda(phys_rec):
    import recomb
    g = load_golden("recomb16.npz")
    he_e = phys_rec.unit("hemf") / phys_rec.unit("hmf") * 0.5
    for i in range(len(g["iso_in_lambdaH"])):
        lam0, gd, tm, nH, T = (float(g[f"iso_in_{k}"][i]) for k in ("lambdaH", "yGdepHI", "time", "nH", "T"))
        lam1, dy = recomb.iso_step(lam0, gd, tm, nH, T, 0.0, he_e, phys_rec.ar_get)
        assert abs(min(1.0, max(0.0, lam1)) - g["iso_out_lambdaH"][i]) < 5e-4
        assert abs(g["iso_in_yGrecHII"][i] + dy - g["iso_out_yGrecHII"][i]) < RTOL_LSODA_ABS


@pytest.mark.parametrize("kind", ["ticks", "ticksthr"])
def test_fixture_rays_are_the_oracle_emission(kind, phys_rec, lte):
    import recomb
    from psphray_b200 import fields
    g = load_golden("recomb16.npz")
    f = fields.make_workload("iliev32", n_side=16, nray=16).field
    pos = np.asarray(f.pos, np.float32).reshape(-1, 3)
    c = _consts(phys_rec)
    nrec = int(g[kind + "_nrec"])
    off = np.concatenate([[0], np.cumsum(g[kind + "_rec_rays_n"])])
    for t in range(2, len(off)):
        b = {k: g[f"{kind}_b_{k}"][t - 1] for k in ("lambdaH", "ie", "ygrec", "mark")}
        rays, em, yg = recomb.emit(b["ygrec"], b["lambdaH"], b["mark"], pos, f.mass, b["ie"], t, nrec, int(g["seed"]),
                                   f.boxsize, c, lte=lte[:2], threshold=float(g["threshold"]))
        gr = g[kind + "_rec_rays"][off[t - 1]:off[t]]
        assert np.array_equal(em, g[kind + "_rec_ipar"][off[t - 1]:off[t]])
        assert np.array_equal(rays, gr)
        # the emitters: marked in the previous tick; their photons leave
        assert np.all(b["mark"][em] == t - 1)
        for p in np.unique(em):
            sel = em == p
            assert np.isclose(rays["Nph"][sel].sum(), float(b["ygrec"][p]) * float(f.mass[p]) * c["H_PER_MASS"],
                              rtol=1e-12)
            assert yg[p] <= 1e-6 * b["ygrec"][p]


def test_fixture_marks_follow_the_hits():
    g = load_golden("recomb16.npz")
    for kind in ("ticks", "ticksthr"):
        a_mark, a_lh, b_mark = g[kind + "_a_mark"], g[kind + "_a_lasthit"], g[kind + "_b_mark"]
        for t in range(1, len(a_mark) + 1):
            new = a_mark[t - 1] == t
            assert new.any()
            # every marked particle was updated this tick; others keep their mark
            assert np.all(a_lh[t - 1][new] == t)
            assert np.array_equal(a_mark[t - 1][~new], b_mark[t - 1][~new])
