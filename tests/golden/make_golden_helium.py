"""Golden vectors for helium and secondary ionisation (psphray.HOnly =
false, psphray.secondaryIonization), from the reference's own code
(oracle/_ref/libpsphray_ref.so and libpsphray_ref_euler.so, `make -C oracle
ref`).

    python tests/golden/make_golden_helium.py

writes tests/golden/helium16.npz:

- Step records before and after step_evolve() with helium (solve.c:170-224,
  LSODA; and step_evolve_euler(), solve.c:225-316), isothermal and not;
- the state after loading the 16^3 uniform field (hydrogen mass fraction
  0.76): the helium fractions and yeMET split off the ye block
  (psystem.c:340-358);
- ticks of that field lit by a corner source with an 8-line 1e5 K blackbody
  (1 to 10 Ry): per tick the state before (lambdaH, lambdaHeI, lambdaHeII,
  ie, lasthit, hits), the tick's rays, the deposits after its deposit()
  (yGdepHI, heat, yGdepHeI, yGdepHeII) and the state after its
  merge_pars() and update_pars(). Three runs: helium isothermal; helium
  with secondary ionisation, not isothermal; hydrogen only (hydrogen mass
  fraction 1) with secondary ionisation, not isothermal;
- not on the spot (case-A recombination): Step records with the three
  species' recombination photons, and ticks of helium, isothermal, with the
  recombination rays of all three species (made by the oracle's
  restatement of the device's emission, oracle/recomb.py, from each tick's
  state) run by the reference's tick phases;
- the explicit build (step_evolve_euler()) with helium, isothermal: ticks
  from the load, the state after each.

The reference keeps its state in globals, so each case runs in a process of
its own.
"""
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

HMF = 0.76
NTICK = 6
NRAY = 16
SEED = 31


def _field(units):
    from psphray_b200 import fields
    return fields.uniform_field(16, SEED, units=units)


def _schedule(units, f):
    from psphray_b200 import fields
    tick_time = 500 * units.MYR / 10000
    e, w = fields.blackbody_bins(units)
    src = [fields.Source(pos=(0.0, 0.0, 0.0), ngamma_dot=5e-2 * 1e50 / units.SEC)]
    return fields.RaySchedule(sources=src, nray=NRAY, tick_time=tick_time, boxsize=f.boxsize, seed=SEED + 1,
                              energies=e, eweights=w), tick_time


def _steps(f, tick_time, seed, n, iso, units):
    from refpy import Step
    rng = np.random.default_rng(seed)
    steps = (Step * n)()
    nH = float(f.rho[0]) * units.H_PER_MASS
    for s in steps:
        s.lambdaH = 10 ** rng.uniform(-4, 0)
        s.lambdaHeI = rng.uniform(0.0, 1.0)
        s.lambdaHeII = rng.uniform(0.0, 1.0 - s.lambdaHeI)
        s.ie = float(f.ie[0]) * (1.0 if iso else 10 ** rng.uniform(0.0, 0.3))
        s.yeMET = 0.0
        s.yGdepHI = 10 ** rng.uniform(-6, -1) if rng.random() < 0.8 else 0.0
        s.yGdepHeI = 10 ** rng.uniform(-6, -1) if rng.random() < 0.5 else 0.0
        s.yGdepHeII = 10 ** rng.uniform(-6, -2) if rng.random() < 0.5 else 0.0
        s.heat = 0.0 if iso else (s.yGdepHI + s.yGdepHeI) * 1e-3 * float(f.ie[0])
        s.time = tick_time * int(rng.integers(1, 200 if iso else 40))
        s.nH = nH
        s.T = 1e4
        s.yGrecHII, s.yGrecHeII, s.yGrecHeIII = rng.uniform(0.0, 0.3, 3)
    return steps


STEP_IN = ["lambdaH", "lambdaHeI", "lambdaHeII", "ie", "yGdepHI", "yGdepHeI", "yGdepHeII", "heat", "time", "nH",
           "T", "yeMET", "yGrecHII", "yGrecHeII", "yGrecHeIII"]
STEP_OUT = ["lambdaH", "lambdaHeI", "lambdaHeII", "ie", "step_remain", "refined", "yGrecHII", "yGrecHeII",
            "yGrecHeIII"]
NREC = 6
REC_SEED = 11


def _case(kind, q):
    from psphray_b200 import api
    from psphray_b200.units import Units
    from refpy import EULER_LIB_PATH, LIB_PATH, Reference
    # hydrogen only: hmf = 1 (with HOnly, helium counts as fully ionised and
    # its electrons' cooling would outrun ie within a tick, which the
    # reference traps, solve.c:137-139)
    units = Units(hmf=1.0 if kind == "h_si" else HMF)
    f = _field(units)
    sch, tick_time = _schedule(units, f)
    out = {}
    if kind in ("iso", "noniso", "euler_iso", "euler_noniso", "rec_iso", "rec_noniso"):
        iso = kind in ("iso", "euler_iso", "rec_iso")
        lib = EULER_LIB_PATH if kind.startswith("euler") else LIB_PATH
        ref = Reference(api.RATES_HUI, units, isothermal=iso, h_only=False, on_the_spot=not kind.startswith("rec"),
                        threads=1, lib_path=lib)
        seed = {"iso": 41, "noniso": 42, "euler_iso": 43, "euler_noniso": 44, "rec_iso": 45, "rec_noniso": 46}[kind]
        steps = _steps(f, tick_time, seed, 192, iso, units)
        for k in STEP_IN:
            out[f"{kind}_in_{k}"] = np.array([getattr(s, k) for s in steps])
        ref.step_evolve(steps)
        for k in STEP_OUT:
            out[f"{kind}_out_{k}"] = np.array([getattr(s, k) for s in steps])
    elif kind == "he_rec":
        _rec_ticks(units, f, sch, tick_time, out)
    elif kind == "he_euler":
        # the explicit build, helium, isothermal: ticks run freely from the
        # load (the photons an early-terminated step leaves stay in yGdep*,
        # loop.c:745-747)
        ref = Reference(api.RATES_HUI, units, isothermal=True, h_only=False, threads=1, lib_path=EULER_LIB_PATH)
        ref.load(f)
        ref.build_tree(8)
        rec = {k: [] for k in ("lambdaH", "lambdaHeI", "lambdaHeII", "ie", "lasthit", "hits")}
        rays_all = []
        for t in range(1, NTICK + 1):
            rays = sch.rays_for_tick(t)
            rays_all.append(rays)
            ref.set_rays(rays, t, tick_time)
            ref.trace(); ref.deposit(); ref.merge(); ref.update()
            s, he = ref.state(), ref.he_state()
            for k in rec:
                rec[k].append(he[k] if k.startswith("lambdaHe") else s[k])
        for k in rec:
            out["he_euler_a_" + k] = np.stack(rec[k])
        out["he_euler_rays"] = np.stack(rays_all)
    else:
        iso = kind == "he_iso"
        h_only = kind == "h_si"
        ref = Reference(api.RATES_HUI, units, isothermal=iso, h_only=h_only, threads=1)
        ref.set_secondary(kind != "he_iso")
        ref.load(f)
        ref.build_tree(8)
        he = ref.he_state()
        p = kind + "_"
        out[p + "load_lambdaHeI"], out[p + "load_lambdaHeII"], out[p + "load_yeMET"] = \
            he["lambdaHeI"], he["lambdaHeII"], he["yeMET"]
        rec = {k: [] for k in ("lambdaH", "lambdaHeI", "lambdaHeII", "ie", "lasthit", "hits")}
        before = {k: [] for k in rec}
        rays_all = []
        dep = {k: [] for k in ("yGdepHI", "heat", "yGdepHeI", "yGdepHeII")}
        for t in range(1, NTICK + 1):
            s, he = ref.state(), ref.he_state()
            for k in rec:
                before[k].append(he[k] if k.startswith("lambdaHe") else s[k])
            rays = sch.rays_for_tick(t)
            rays_all.append(rays)
            ref.set_rays(rays, t, tick_time)
            ref.trace(); ref.deposit()
            s, he = ref.state(), ref.he_state()
            for k in dep:
                dep[k].append(he[k] if k.startswith("yGdepHe") else s[k])
            ref.merge(); ref.update()
            s, he = ref.state(), ref.he_state()
            for k in rec:
                rec[k].append(he[k] if k.startswith("lambdaHe") else s[k])
        for k in rec:
            out[p + "b_" + k] = np.stack(before[k])
            out[p + "a_" + k] = np.stack(rec[k])
        out[p + "rays"] = np.stack(rays_all)
        for k in dep:
            out[p + "d_" + k] = np.stack(dep[k])
    out["tick_time"] = np.float64(tick_time)
    q.put(out)


def _rec_ticks(units, f, sch, tick_time, out):
    """Helium, isothermal, not on the spot: the ticks with the recombination
    rays of all three species (oracle/recomb.py) from each tick's state."""
    import recomb
    from psphray_b200 import api
    from refpy import Reference
    phys = api.Physics(units, isothermal=True, on_the_spot=False, h_only=False)
    c = {k: phys.unit(k) for k in ("HI_ENERGY", "HEI_ENERGY", "HEII_ENERGY", "BOLTZMANN", "H_PER_MASS",
                                   "HE_PER_MASS", "MPROTON_OVER_BOLTZMANN", "hmf", "hemf")}
    ltes = [recomb.lte_table(c[th], c["BOLTZMANN"], (lambda sp: (lambda e: phys.xs_get(sp, e)))(sp))
            for th, sp in zip(recomb.THRESHOLDS, ("HI", "HeI", "HeII"))]
    ref = Reference(api.RATES_HUI, units, isothermal=True, h_only=False, on_the_spot=False, threads=1)
    ref.load(f)
    ref.build_tree(8)
    pos = np.asarray(f.pos, np.float32).reshape(-1, 3)
    mass = np.asarray(f.mass, np.float32)
    mark = np.full(f.n, -1, np.int32)
    keys = ("lambdaH", "lambdaHeI", "lambdaHeII", "ie", "lasthit", "hits", "yg0", "yg1", "yg2", "mark")
    b, a = {k: [] for k in keys}, {k: [] for k in keys}
    rays_src, rays_rec, rec_ipar, rec_type = [], [], [], []

    def snap(dst):
        s, he, yg = ref.state(), ref.he_state(), ref.ygrec3()
        vals = dict(lambdaH=s["lambdaH"], lambdaHeI=he["lambdaHeI"], lambdaHeII=he["lambdaHeII"], ie=s["ie"],
                    lasthit=s["lasthit"], hits=s["hits"], yg0=yg[0], yg1=yg[1], yg2=yg[2], mark=mark.copy())
        for k in keys:
            dst[k].append(vals[k])
        return vals
    R = sch.nray
    for t in range(1, NTICK + 1):
        v = snap(b)
        src = sch.rays_for_tick(t)
        if t > 1:
            rr, em, ty, ygs = recomb.emit([v["yg0"], v["yg1"], v["yg2"]], v["lambdaH"], mark, pos, mass, v["ie"], t,
                                          NREC, REC_SEED, f.boxsize, c, lte=ltes, l1=v["lambdaHeI"],
                                          l2=v["lambdaHeII"], types=True)
            ref.set_ygrec3(ygs)
        else:
            rr, em, ty = np.zeros(0, src.dtype), np.zeros(0, np.int64), np.zeros(0, np.int32)
        ref.set_rays(np.concatenate([src, rr]), t, tick_time)
        ref.trace(); ref.deposit(); ref.merge(); ref.update()
        for i in range(R + (1 if len(rr) else 0)):
            mark[ref.ray_hits(i)[0]] = t
        snap(a)
        rays_src.append(src); rays_rec.append(rr); rec_ipar.append(em); rec_type.append(ty)
    for k in keys:
        out["he_rec_b_" + k] = np.stack(b[k])
        out["he_rec_a_" + k] = np.stack(a[k])
    out["he_rec_rays"] = np.stack(rays_src)
    out["he_rec_rec_rays"] = np.concatenate(rays_rec)
    out["he_rec_rec_ipar"] = np.concatenate(rec_ipar)
    out["he_rec_rec_type"] = np.concatenate(rec_type)
    out["he_rec_rec_n"] = np.array([len(x) for x in rays_rec], np.int64)
    out["he_rec_nrec"] = np.int64(NREC)
    out["he_rec_seed"] = np.int64(REC_SEED)


def main():
    ctx = mp.get_context("spawn")
    out = {"hmf": np.float64(HMF)}
    for kind in ("iso", "noniso", "euler_iso", "euler_noniso", "rec_iso", "rec_noniso", "he_iso", "he_si", "h_si",
                 "he_rec", "he_euler"):
        q = ctx.Queue()
        p = ctx.Process(target=_case, args=(kind, q))
        p.start()
        got = None
        while got is None:
            try:
                got = q.get(timeout=5)
            except Exception:
                if not p.is_alive():
                    raise RuntimeError(f"case {kind} died (exit code {p.exitcode})")
        out.update(got)
        p.join()
        assert p.exitcode == 0, kind
    np.savez_compressed(os.path.join(HERE, "helium16.npz"), **out)
    print("wrote", os.path.join(HERE, "helium16.npz"), sorted(out))


if __name__ == "__main__":
    main()
