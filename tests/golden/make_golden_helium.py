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
  merge_pars() and update_pars(). Three runs: helium
  isothermal; helium with secondary ionisation, not isothermal; hydrogen
  only (hydrogen mass fraction 1) with secondary ionisation, not
  isothermal.

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
    return steps


STEP_IN = ["lambdaH", "lambdaHeI", "lambdaHeII", "ie", "yGdepHI", "yGdepHeI", "yGdepHeII", "heat", "time", "nH",
           "T", "yeMET"]
STEP_OUT = ["lambdaH", "lambdaHeI", "lambdaHeII", "ie", "step_remain", "refined"]


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
    if kind in ("iso", "noniso", "euler_iso", "euler_noniso"):
        iso = kind in ("iso", "euler_iso")
        lib = EULER_LIB_PATH if kind.startswith("euler") else LIB_PATH
        ref = Reference(api.RATES_HUI, units, isothermal=iso, h_only=False, threads=1, lib_path=lib)
        seed = {"iso": 41, "noniso": 42, "euler_iso": 43, "euler_noniso": 44}[kind]
        steps = _steps(f, tick_time, seed, 192, iso, units)
        for k in STEP_IN:
            out[f"{kind}_in_{k}"] = np.array([getattr(s, k) for s in steps])
        ref.step_evolve(steps)
        for k in STEP_OUT:
            out[f"{kind}_out_{k}"] = np.array([getattr(s, k) for s in steps])
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


def main():
    ctx = mp.get_context("spawn")
    out = {"hmf": np.float64(HMF)}
    for kind in ("iso", "noniso", "euler_iso", "euler_noniso", "he_iso", "he_si", "h_si"):
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
