"""Runs not on the spot (psphray.onTheSpot = false) on the device:
case-A recombination, the recombination photons yGrecHII and the
recombination rays, against tests/golden/recomb16.npz (the reference's own
step_evolve() and tick phases, tests/golden/make_golden_recomb.py) and the
oracle's restatements (oracle/recomb.py).

Tolerances: against the reference's LSODA (rtol 1e-4, atol 1e-7), whose own
error against a tight implicit integration is up to 3e-5 in lambdaH, 1.4e-3
in ie and 1.1e-5 in yGrecHII on these steps; against the oracle's closed
form 1e-12 in lambdaH (1e-9 of the yGrecHII gained), and against its tight
integration the device integrators' tolerances (rtol 1e-6, 1e-5 for the
stiff finish). Ray emission is bit-exact with the oracle's
restatement (directions to a float rounding).
"""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

LAM_LSODA, IE_LSODA, YG_LSODA = 5e-4, 3e-3, 3e-5


def _consts(phys):
    return {k: phys.unit(k) for k in ("HI_ENERGY", "BOLTZMANN", "H_PER_MASS", "MPROTON_OVER_BOLTZMANN", "hmf", "hemf")}


def _steps(g, kind):
    from psphray_b200 import api
    n = len(g[f"{kind}_in_lambdaH"])
    steps = np.zeros(n, api.STEP_DTYPE)
    for k in ("lambdaH", "ie", "yGdepHI", "heat", "time", "nH", "T", "yeMET", "yGrecHII"):
        steps[k] = g[f"{kind}_in_{k}"]
    return steps


def test_step_evolve_iso_not_on_the_spot(gpu_ctx, units):
    import recomb
    from psphray_b200 import api
    g = load_golden("recomb16.npz")
    phys = api.Physics(units, isothermal=True, on_the_spot=False)
    gpu_ctx.set_physics(phys)
    steps = _steps(g, "iso")
    out = gpu_ctx.step_evolve(steps.copy())
    he_e = phys.unit("hemf") / phys.unit("hmf") * 0.5
    for i, s in enumerate(steps):
        lam, dy = recomb.iso_step(s["lambdaH"], s["yGdepHI"], s["time"], s["nH"], s["T"], s["yeMET"], he_e,
                                  phys.ar_get)
        assert abs(out["lambdaH"][i] - min(1.0, max(0.0, lam))) < 1e-12
        assert abs(out["yGrecHII"][i] - (s["yGrecHII"] + dy)) <= 1e-9 * abs(dy) + 1e-15
    assert np.max(np.abs(out["lambdaH"] - g["iso_out_lambdaH"])) < LAM_LSODA
    assert np.max(np.abs(out["yGrecHII"] - g["iso_out_yGrecHII"])) < YG_LSODA


def test_step_evolve_noniso_not_on_the_spot(gpu_ctx, units):
    import recomb
    from psphray_b200 import api
    g = load_golden("recomb16.npz")
    phys = api.Physics(units, isothermal=False, on_the_spot=False)
    gpu_ctx.set_physics(phys)
    steps = _steps(g, "noniso")
    out = gpu_ctx.step_evolve(steps.copy())
    c = _consts(phys)
    for i in range(0, len(steps), 8):
        s = steps[i]
        lam, ie, yg = recomb.noniso_step(s["lambdaH"], s["ie"], s["yGdepHI"], s["heat"], s["time"], s["nH"],
                                         s["yeMET"], s["yGrecHII"], c, phys.ar_get)
        assert abs(out["lambdaH"][i] - lam) < 1e-5
        assert abs(out["ie"][i] / ie - 1) < 1e-4
        assert abs(out["yGrecHII"][i] - yg) < 3e-7
    assert np.max(np.abs(out["lambdaH"] - g["noniso_out_lambdaH"])) < LAM_LSODA
    assert np.max(np.abs(out["ie"] / g["noniso_out_ie"] - 1)) < IE_LSODA
    assert np.max(np.abs(out["yGrecHII"] - g["noniso_out_yGrecHII"])) < YG_LSODA


def _rec_ctx(units, g, kind):
    from psphray_b200 import api, fields
    w = fields.make_workload("iliev32", n_side=16, nray=16)
    phys = api.Physics(units, isothermal=True, on_the_spot=False)
    c = api.Context(0)
    c.set_physics(phys)
    c.load(w.field)
    c.build_tree(8)
    nrec = int(g[kind + "_nrec"])
    c.set_recombination(nrec=nrec, threshold=float(g["threshold"]), disable_lte=False, seed=int(g["seed"]))
    return c, w


@pytest.mark.parametrize("kind", ["ticks", "ticksthr"])
def test_ticks_with_recombination_rays(units, kind):
    """Each tick from the reference's state before it: the device's
    recombination rays are the oracle's, and the state after the tick is
    the reference's (trace, deposit, merge and update of the source and
    recombination rays together)."""
    g = load_golden("recomb16.npz")
    ctx, w = _rec_ctx(units, g, kind)
    try:
        off = np.concatenate([[0], np.cumsum(g[kind + "_rec_rays_n"])])
        R = w.schedule.nray
        tt = float(g["tick_time"])
        nt = len(off) - 1
        for t in range(1, nt + 1):
            b = {k: g[f"{kind}_b_{k}"][t - 1] for k in ("lambdaH", "ie", "lasthit", "hits", "ygrec", "mark")}
            ctx.set_state(lambdaH=b["lambdaH"], ie=b["ie"], lasthit=b["lasthit"])
            ctx.set_hits(b["hits"])
            ctx.set_rec_state(b["ygrec"], b["mark"])
            st = ctx.run_ticks(g[kind + "_src_rays"][t - 1], R, 1, t, tt)
            rays, ipar = ctx.rec_rays()
            gr, gi = g[kind + "_rec_rays"][off[t - 1]:off[t]], g[kind + "_rec_ipar"][off[t - 1]:off[t]]
            assert st["rec_rays"] == len(gr)
            assert np.array_equal(ipar, gi), t
            assert np.array_equal(rays["s"], gr["s"]) and np.array_equal(rays["length"], gr["length"])
            assert np.array_equal(rays["Nph"], gr["Nph"]) and np.array_equal(rays["freq"], gr["freq"])
            assert np.max(np.abs(rays["dir"] - gr["dir"]), initial=0.0) < 1e-6
            a = ctx.state()
            yg, mark = ctx.rec_state()
            assert np.array_equal(a["hits"], g[kind + "_a_hits"][t - 1]), t
            assert np.array_equal(a["lasthit"], g[kind + "_a_lasthit"][t - 1]), t
            assert np.array_equal(mark, g[kind + "_a_mark"][t - 1]), t
            assert np.max(np.abs(a["lambdaH"] - g[kind + "_a_lambdaH"][t - 1])) < LAM_LSODA
            assert np.max(np.abs(a["ie"] / g[kind + "_a_ie"][t - 1] - 1)) < IE_LSODA
            assert np.max(np.abs(yg - g[kind + "_a_ygrec"][t - 1])) < YG_LSODA
    finally:
        ctx.close()


def test_batched_ticks_equal_single_ticks(units):
    """K ticks in one call run tick by tick on the device: the same state as
    K calls of one tick; the photons emitted leave yGrecHII."""
    g = load_golden("recomb16.npz")
    src = g["ticks_src_rays"]
    R, nt, tt = src.shape[1], src.shape[0], float(g["tick_time"])
    a, _ = _rec_ctx(units, g, "ticks")
    b, _ = _rec_ctx(units, g, "ticks")
    try:
        sa = a.run_ticks(src.reshape(-1), R, nt, 1, tt)
        nrays = 0
        for t in range(1, nt + 1):
            nrays += b.run_ticks(src[t - 1], R, 1, t, tt)["rec_rays"]
        assert sa["rec_rays"] == nrays == 24 * (nt - 1)
        assert sa["rec_photons"] > 0
        x, y = a.state(), b.state()
        for k in ("lambdaH", "ie", "hits", "lasthit"):
            assert np.array_equal(x[k], y[k]), k
        assert all(np.array_equal(u, v) for u, v in zip(a.rec_state(), b.rec_state()))
    finally:
        a.close()
        b.close()
