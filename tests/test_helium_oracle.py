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
