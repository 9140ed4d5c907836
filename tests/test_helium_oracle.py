"""The helium / secondary-ionisation oracle (oracle/helium.py) and the
product's secondary-ionisation table (psg_secion_table_build) against the
reference's own code (secion.c built into the harness) and the golden
fixture tests/golden/helium16.npz (tests/golden/make_golden_helium.py)."""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden

HMF = 0.76


def _table(phys):
    from psphray_b200 import api
    out = np.zeros(3 * 4096 * 1024)
    assert api.lib().psg_secion_table_build(C.byref(phys.cu), out.ctypes.data) == 0
    return out.reshape(3, 4096, 1024)


def test_secion_table_and_lookup_vs_reference(reference, phys):
    import helium
    reference.set_secondary(True)
    tab = _table(phys)
    ev = phys.unit("EV")
    rng = np.random.default_rng(4)
    step1 = (200 * ev - 10 * ev) / 4096
    for _ in range(2000):        # the grid itself
        c, i, j = rng.integers(0, 3), rng.integers(0, 4096), rng.integers(0, 1024)
        r = reference.secion_get(int(c), 10 * ev + i * step1, -8 + j * 8 / 1024)
        assert abs(tab[c, i, j] - r) <= 1e-12 * abs(r) + 1e-300
    for _ in range(3000):        # lookups inside and outside the table
        c = int(rng.integers(0, 3))
        E = rng.uniform(-5, 250) * ev
        y = rng.uniform(-9, 0.0)
        r = reference.secion_get(c, E, y)
        assert abs(helium.secion_get(tab, c, E, y, ev) - r) <= 1e-11 * abs(r) + 1e-15


def test_load_split_matches_reference():
    import helium
    from psphray_b200 import fields
    from psphray_b200.units import Units
    g = load_golden("helium16.npz")
    f = fields.uniform_field(16, 31, units=Units(hmf=HMF))
    l1, l2, ym = helium.load_split(f.xHI, f.ye, HMF)
    for k in ("he_iso", "he_si"):
        assert np.array_equal(l1, g[k + "_load_lambdaHeI"]) and np.array_equal(l2, g[k + "_load_lambdaHeII"])
        assert np.array_equal(ym, g[k + "_load_yeMET"])


@pytest.mark.parametrize("kind", ["iso", "noniso"])
def test_helium_step_vs_lsoda(kind, units):
    import helium
    from psphray_b200 import api
    from psphray_b200.units import Units
    g = load_golden("helium16.npz")
    iso = kind == "iso"
    phys = api.Physics(Units(hmf=HMF), isothermal=iso, h_only=False)
    c = {k: phys.unit(k) for k in ("H_PER_MASS", "MPROTON_OVER_BOLTZMANN", "hmf", "hemf")}
    for i in range(0, len(g[kind + "_in_lambdaH"]), 6):
        s = {k: float(g[f"{kind}_in_{k}"][i]) for k in ("lambdaH", "lambdaHeI", "lambdaHeII", "ie", "yGdepHI",
                                                         "yGdepHeI", "yGdepHeII", "heat", "time", "nH", "T", "yeMET")}
        x = helium.he_step((s["lambdaH"], s["lambdaHeI"], s["lambdaHeII"], s["ie"]), s["yeMET"], s["yGdepHI"],
                           s["yGdepHeI"], s["yGdepHeII"], s["heat"], s["time"], s["nH"], s["T"], c, phys.ar_get, iso)
        for j, k in enumerate(("lambdaH", "lambdaHeI", "lambdaHeII")):
            assert abs(x[j] - g[f"{kind}_out_{k}"][i]) < 1e-4, (i, k)
        assert abs(x[3] / g[f"{kind}_out_ie"][i] - 1) < 3e-3


@pytest.mark.parametrize("kind", ["rec_iso", "rec_noniso"])
def test_helium_step_not_on_the_spot_vs_lsoda(kind):
    """Case-A helium with the three species' recombination photons."""
    import helium
    from psphray_b200 import api
    from psphray_b200.units import Units
    g = load_golden("helium16.npz")
    iso = kind == "rec_iso"
    phys = api.Physics(Units(hmf=HMF), isothermal=iso, h_only=False, on_the_spot=False)
    c = {k: phys.unit(k) for k in ("H_PER_MASS", "MPROTON_OVER_BOLTZMANN", "hmf", "hemf")}
    for i in range(0, len(g[kind + "_in_lambdaH"]), 6):
        s = {k: float(g[f"{kind}_in_{k}"][i]) for k in ("lambdaH", "lambdaHeI", "lambdaHeII", "ie", "yGdepHI",
                                                         "yGdepHeI", "yGdepHeII", "heat", "time", "nH", "T", "yeMET",
                                                         "yGrecHII", "yGrecHeII", "yGrecHeIII")}
        x = helium.he_step((s["lambdaH"], s["lambdaHeI"], s["lambdaHeII"], s["ie"]), s["yeMET"], s["yGdepHI"],
                           s["yGdepHeI"], s["yGdepHeII"], s["heat"], s["time"], s["nH"], s["T"], c, phys.ar_get, iso,
                           on_the_spot=False, rec0=(s["yGrecHII"], s["yGrecHeII"], s["yGrecHeIII"]))
        for j, k in enumerate(("lambdaH", "lambdaHeI", "lambdaHeII")):
            assert abs(x[j] - g[f"{kind}_out_{k}"][i]) < 1e-4, (i, k)
        assert abs(x[3] / g[f"{kind}_out_ie"][i] - 1) < 3e-3
        for j, k in enumerate(("yGrecHII", "yGrecHeII", "yGrecHeIII")):
            assert abs(x[4 + j] - g[f"{kind}_out_{k}"][i]) < 3e-5, (i, k)


def test_fixture_helium_recombination_rays_are_the_oracle_emission():
    import recomb
    from psphray_b200 import api, fields
    from psphray_b200.units import Units
    g = load_golden("helium16.npz")
    units = Units(hmf=HMF)
    f = fields.uniform_field(16, 31, units=units)
    phys = api.Physics(units, isothermal=True, on_the_spot=False, h_only=False)
    c = {k: phys.unit(k) for k in ("HI_ENERGY", "HEI_ENERGY", "HEII_ENERGY", "BOLTZMANN", "H_PER_MASS",
                                   "HE_PER_MASS", "MPROTON_OVER_BOLTZMANN", "hmf", "hemf")}
    ltes = [recomb.lte_table(c[th], c["BOLTZMANN"], (lambda sp: (lambda e: phys.xs_get(sp, e)))(sp))
            for th, sp in zip(recomb.THRESHOLDS, ("HI", "HeI", "HeII"))]
    pos = np.asarray(f.pos, np.float32).reshape(-1, 3)
    off = np.concatenate([[0], np.cumsum(g["he_rec_rec_n"])])
    for t in range(2, len(off)):
        b = {k: g["he_rec_b_" + k][t - 1] for k in ("lambdaH", "lambdaHeI", "lambdaHeII", "ie", "yg0", "yg1", "yg2",
                                                     "mark")}
        rays, em, ty, ygs = recomb.emit([b["yg0"], b["yg1"], b["yg2"]], b["lambdaH"], b["mark"], pos, f.mass, b["ie"],
                                        t, int(g["he_rec_nrec"]), int(g["he_rec_seed"]), f.boxsize, c, lte=ltes,
                                        l1=b["lambdaHeI"], l2=b["lambdaHeII"], types=True)
        sl = slice(off[t - 1], off[t])
        assert np.array_equal(rays, g["he_rec_rec_rays"][sl])
        assert np.array_equal(em, g["he_rec_rec_ipar"][sl]) and np.array_equal(ty, g["he_rec_rec_type"][sl])
        assert np.all(b["mark"][em] == t - 1)
