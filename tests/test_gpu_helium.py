"""Helium (psphray.HOnly = false) and secondary ionisation on the device,
against tests/golden/helium16.npz (the reference's own step_evolve() and
tick phases, tests/golden/make_golden_helium.py) and the oracle's tight
integration of the helium step (oracle/helium.py).

Tolerances: the reference's LSODA (rtol 1e-4, atol 1e-7) differs from a
tight implicit integration of the same equations by up to 3.5e-5 in the
fractions and 1.2e-3 in ie on the Step records, and by up to 0.7% in ie on
strongly heated particles of the ticks; the device integrator (rtol 1e-6;
1e-5 in the stiff finish) is checked against the tight integration to
1e-5 (fractions) and 1e-4 (ie), and against LSODA to 1e-4 (fractions) and
3e-3 (ie) wherever LSODA itself is that close. Hit counts and lasthit are
exact."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

HMF = 0.76
STEP_KEYS = ("lambdaH", "lambdaHeI", "lambdaHeII", "ie", "yGdepHI", "yGdepHeI", "yGdepHeII", "heat", "time", "nH",
             "T", "yeMET")


def _steps(g, kind):
    from psphray_b200 import api
    n = len(g[f"{kind}_in_lambdaH"])
    steps = np.zeros(n, api.STEP_DTYPE)
    for k in STEP_KEYS:
        steps[k] = g[f"{kind}_in_{k}"]
    return steps


@pytest.mark.parametrize("kind", ["iso", "noniso"])
def test_step_evolve_helium(gpu_ctx, kind):
    import helium
    from psphray_b200 import api
    from psphray_b200.units import Units
    g = load_golden("helium16.npz")
    iso = kind == "iso"
    phys = api.Physics(Units(hmf=HMF), isothermal=iso, h_only=False)
    gpu_ctx.set_physics(phys)
    steps = _steps(g, kind)
    out = gpu_ctx.step_evolve(steps.copy())
    c = {k: phys.unit(k) for k in ("H_PER_MASS", "MPROTON_OVER_BOLTZMANN", "hmf", "hemf")}
    for i in range(0, len(steps), 6):
        s = steps[i]
        x = helium.he_step((s["lambdaH"], s["lambdaHeI"], s["lambdaHeII"], s["ie"]), s["yeMET"], s["yGdepHI"],
                           s["yGdepHeI"], s["yGdepHeII"], s["heat"], s["time"], s["nH"], s["T"], c, phys.ar_get, iso)
        for j, k in enumerate(("lambdaH", "lambdaHeI", "lambdaHeII")):
            assert abs(out[k][i] - x[j]) < 1e-5, (i, k)
        assert abs(out["ie"][i] / x[3] - 1) < 1e-5
    for k in ("lambdaH", "lambdaHeI", "lambdaHeII"):
        assert np.max(np.abs(out[k] - g[f"{kind}_out_{k}"])) < 1e-4, k
    assert np.max(np.abs(out["ie"] / g[f"{kind}_out_ie"] - 1)) < 3e-3


@pytest.mark.parametrize("kind", ["euler_iso", "euler_noniso"])
def test_step_evolve_helium_euler(gpu_ctx, kind):
    from psphray_b200 import api
    from psphray_b200.units import Units
    g = load_golden("helium16.npz")
    phys = api.Physics(Units(hmf=HMF), isothermal=kind == "euler_iso", h_only=False, euler=True)
    gpu_ctx.set_physics(phys)
    out = gpu_ctx.step_evolve(_steps(g, kind))
    for k in ("lambdaH", "lambdaHeI", "lambdaHeII"):
        assert np.max(np.abs(out[k] - g[f"{kind}_out_{k}"])) < 1e-6, k
    assert np.max(np.abs(out["ie"] / g[f"{kind}_out_ie"] - 1)) < 1e-6
    assert np.array_equal(out["refined"], g[f"{kind}_out_refined"])
    assert np.array_equal(out["step_remain"], g[f"{kind}_out_step_remain"])


def _tight(phys, f, b, d, p, t, tt, iso, h_only):
    """The particle's step integrated tightly from the reference's state
    and deposits of the tick (oracle/helium.py)."""
    import helium
    c = {k: phys.unit(k) for k in ("H_PER_MASS", "MPROTON_OVER_BOLTZMANN", "hmf", "hemf")}
    x0 = (b["lambdaH"][p], b["lambdaHeI"][p], b["lambdaHeII"][p], float(b["ie"][p]))
    return helium.he_step(x0, 0.0, float(d["yGdepHI"][p]), float(d["yGdepHeI"][p]), float(d["yGdepHeII"][p]),
                          float(d["heat"][p]), (t - b["lasthit"][p]) * tt, float(f.rho[p]) * c["H_PER_MASS"], 1e4, c,
                          phys.ar_get, iso, h_only=h_only)


@pytest.mark.parametrize("kind", ["he_iso", "he_si", "h_si"])
def test_ticks_helium_and_secondary(kind):
    """Each tick from the reference's state before it: hits and lasthit
    exact; the fractions and ie to LSODA's tolerance, or, where the
    reference's LSODA itself is off by more (strong secondary heating: up
    to 0.7% in ie), to 1e-4 of a tight integration of the reference's own
    deposits."""
    from psphray_b200 import api, fields
    from psphray_b200.units import Units
    g = load_golden("helium16.npz")
    units = Units(hmf=1.0 if kind == "h_si" else HMF)
    f = fields.uniform_field(16, 31, units=units)
    iso = kind == "he_iso"
    phys = api.Physics(units, isothermal=iso, h_only=kind == "h_si", secondary_ionization=kind != "he_iso")
    ctx = api.Context(0)
    try:
        ctx.set_physics(phys)
        ctx.load(f)
        ctx.build_tree(8)
        he = ctx.he_state()
        assert np.array_equal(he["lambdaHeI"], g[kind + "_load_lambdaHeI"])
        assert np.array_equal(he["lambdaHeII"], g[kind + "_load_lambdaHeII"])
        assert np.array_equal(he["yeMET"], g[kind + "_load_yeMET"])
        rays = g[kind + "_rays"]
        tt = float(g["tick_time"])
        for t in range(1, rays.shape[0] + 1):
            b = {k: g[f"{kind}_b_{k}"][t - 1] for k in ("lambdaH", "lambdaHeI", "lambdaHeII", "ie", "lasthit", "hits")}
            d = {k: g[f"{kind}_d_{k}"][t - 1] for k in ("yGdepHI", "heat", "yGdepHeI", "yGdepHeII")}
            ctx.set_state(lambdaH=b["lambdaH"], ie=b["ie"], lasthit=b["lasthit"])
            ctx.set_hits(b["hits"])
            ctx.set_he_state(b["lambdaHeI"], b["lambdaHeII"])
            ctx.run_ticks(rays[t - 1], rays.shape[1], 1, t, tt)
            a, he = ctx.state(), ctx.he_state()
            dev = {"lambdaH": a["lambdaH"], "lambdaHeI": he["lambdaHeI"], "lambdaHeII": he["lambdaHeII"], "ie": a["ie"]}
            assert np.array_equal(a["hits"], g[kind + "_a_hits"][t - 1]), t
            assert np.array_equal(a["lasthit"], g[kind + "_a_lasthit"][t - 1]), t
            off = np.zeros(f.n, bool)
            for k in ("lambdaH", "lambdaHeI", "lambdaHeII"):
                off |= np.abs(dev[k] - g[f"{kind}_a_{k}"][t - 1]) >= 1e-4
            off |= np.abs(dev["ie"] / g[kind + "_a_ie"][t - 1] - 1) >= 3e-3
            assert off.sum() <= 8, (t, off.sum())
            for p in np.nonzero(off)[0]:
                x = _tight(phys, f, b, d, p, t, tt, iso, kind == "h_si")
                for j, k in enumerate(("lambdaH", "lambdaHeI", "lambdaHeII")):
                    assert abs(dev[k][p] - x[j]) < 1e-5, (t, p, k)
                assert abs(dev["ie"][p] / x[3] - 1) < 1e-4, (t, p)
    finally:
        ctx.close()


@pytest.mark.parametrize("kind", ["rec_iso", "rec_noniso"])
def test_step_evolve_helium_not_on_the_spot(gpu_ctx, kind):
    """Case-A helium with the three species' recombination photons."""
    import helium
    from psphray_b200 import api
    from psphray_b200.units import Units
    g = load_golden("helium16.npz")
    iso = kind == "rec_iso"
    phys = api.Physics(Units(hmf=HMF), isothermal=iso, h_only=False, on_the_spot=False)
    gpu_ctx.set_physics(phys)
    steps = _steps(g, kind)
    for k in ("yGrecHII", "yGrecHeII", "yGrecHeIII"):
        steps[k] = g[f"{kind}_in_{k}"]
    out = gpu_ctx.step_evolve(steps.copy())
    c = {k: phys.unit(k) for k in ("H_PER_MASS", "MPROTON_OVER_BOLTZMANN", "hmf", "hemf")}
    recs = ("yGrecHII", "yGrecHeII", "yGrecHeIII")
    for i in range(0, len(steps), 6):
        s = steps[i]
        x = helium.he_step((s["lambdaH"], s["lambdaHeI"], s["lambdaHeII"], s["ie"]), s["yeMET"], s["yGdepHI"],
                           s["yGdepHeI"], s["yGdepHeII"], s["heat"], s["time"], s["nH"], s["T"], c, phys.ar_get, iso,
                           on_the_spot=False, rec0=tuple(s[k] for k in recs))
        for j, k in enumerate(("lambdaH", "lambdaHeI", "lambdaHeII")):
            assert abs(out[k][i] - x[j]) < 1e-5, (i, k)
        assert abs(out["ie"][i] / x[3] - 1) < 1e-4
        for j, k in enumerate(recs):
            assert abs(out[k][i] - x[4 + j]) < 3e-7, (i, k)
    for k in ("lambdaH", "lambdaHeI", "lambdaHeII"):
        assert np.max(np.abs(out[k] - g[f"{kind}_out_{k}"])) < 1e-4, k
    assert np.max(np.abs(out["ie"] / g[f"{kind}_out_ie"] - 1)) < 3e-3
    for k in recs:
        assert np.max(np.abs(out[k] - g[f"{kind}_out_{k}"])) < 3e-5, k


def test_ticks_helium_recombination_rays():
    """Helium not on the spot, each tick from the reference's state before
    it: the recombination rays of the three species are the oracle's (the
    same emitters, types, photons and energies), hits, lasthit and emitter
    marks exact, the fractions and yGrec to LSODA's tolerance."""
    from psphray_b200 import api, fields
    from psphray_b200.units import Units
    g = load_golden("helium16.npz")
    units = Units(hmf=HMF)
    f = fields.uniform_field(16, 31, units=units)
    phys = api.Physics(units, isothermal=True, h_only=False, on_the_spot=False)
    ctx = api.Context(0)
    try:
        ctx.set_physics(phys)
        ctx.load(f)
        ctx.build_tree(8)
        ctx.set_recombination(nrec=int(g["he_rec_nrec"]), seed=int(g["he_rec_seed"]))
        rays = g["he_rec_rays"]
        off = np.concatenate([[0], np.cumsum(g["he_rec_rec_n"])])
        tt = float(g["tick_time"])
        for t in range(1, rays.shape[0] + 1):
            b = {k: g["he_rec_b_" + k][t - 1] for k in ("lambdaH", "lambdaHeI", "lambdaHeII", "ie", "lasthit", "hits",
                                                         "yg0", "yg1", "yg2", "mark")}
            ctx.set_state(lambdaH=b["lambdaH"], ie=b["ie"], lasthit=b["lasthit"])
            ctx.set_hits(b["hits"])
            ctx.set_he_state(b["lambdaHeI"], b["lambdaHeII"], b["yg1"], b["yg2"])
            ctx.set_rec_state(b["yg0"], b["mark"])
            ctx.run_ticks(rays[t - 1], rays.shape[1], 1, t, tt)
            rr, ipar, typ = ctx.rec_rays(types=True)
            sl = slice(off[t - 1], off[t])
            gr = g["he_rec_rec_rays"][sl]
            assert np.array_equal(ipar, g["he_rec_rec_ipar"][sl]) and np.array_equal(typ, g["he_rec_rec_type"][sl])
            assert np.array_equal(rr["s"], gr["s"]) and np.array_equal(rr["Nph"], gr["Nph"])
            assert np.array_equal(rr["freq"], gr["freq"]) and np.array_equal(rr["length"], gr["length"])
            assert np.max(np.abs(rr["dir"] - gr["dir"]), initial=0.0) < 1e-6
            a, he = ctx.state(), ctx.he_state()
            yg0, mark = ctx.rec_state()
            assert np.array_equal(a["hits"], g["he_rec_a_hits"][t - 1]), t
            assert np.array_equal(a["lasthit"], g["he_rec_a_lasthit"][t - 1]), t
            assert np.array_equal(mark, g["he_rec_a_mark"][t - 1]), t
            assert np.max(np.abs(a["lambdaH"] - g["he_rec_a_lambdaH"][t - 1])) < 1e-4, t
            for k in ("lambdaHeI", "lambdaHeII"):
                assert np.max(np.abs(he[k] - g["he_rec_a_" + k][t - 1])) < 1e-4, (t, k)
            for mine, k in ((yg0, "yg0"), (he["yGrecHeII"], "yg1"), (he["yGrecHeIII"], "yg2")):
                assert np.max(np.abs(mine - g["he_rec_a_" + k][t - 1])) < 3e-5, (t, k)
    finally:
        ctx.close()


def test_ticks_helium_euler():
    """The explicit solver with helium over six ticks from the load: the
    photons an early-terminated step leaves carried to the next update for
    each species (loop.c:745-747); hits and lasthit exact, the fractions
    within 2e-5 of the reference's explicit build."""
    from psphray_b200 import api, fields
    from psphray_b200.units import Units
    g = load_golden("helium16.npz")
    units = Units(hmf=HMF)
    f = fields.uniform_field(16, 31, units=units)
    phys = api.Physics(units, isothermal=True, h_only=False, euler=True)
    ctx = api.Context(0)
    try:
        ctx.set_physics(phys)
        ctx.load(f)
        ctx.build_tree(8)
        rays = g["he_euler_rays"]
        tt = float(g["tick_time"])
        for t in range(1, rays.shape[0] + 1):
            ctx.run_ticks(rays[t - 1], rays.shape[1], 1, t, tt)
            a, he = ctx.state(), ctx.he_state()
            assert np.array_equal(a["hits"], g["he_euler_a_hits"][t - 1]), t
            assert np.array_equal(a["lasthit"], g["he_euler_a_lasthit"][t - 1]), t
            assert np.max(np.abs(a["lambdaH"] - g["he_euler_a_lambdaH"][t - 1])) < 2e-5, t
            for k in ("lambdaHeI", "lambdaHeII"):
                assert np.max(np.abs(he[k] - g["he_euler_a_" + k][t - 1])) < 2e-5, (t, k)
            assert np.max(np.abs(a["ie"] / g["he_euler_a_ie"][t - 1] - 1)) < 1e-4, t
    finally:
        ctx.close()
