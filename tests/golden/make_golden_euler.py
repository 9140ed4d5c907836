"""Golden vectors for the explicit solver (step_evolve_euler(), solve.c:225-316)
from the reference's own code built without USE_LSODA
(oracle/_ref/libpsphray_ref_euler.so, `make -C oracle ref`).

    python tests/golden/make_golden_euler.py

writes tests/golden/euler16.npz: Step records before and after
step_evolve() (isothermal and not), and the particle state over 20 ticks
of the 16^3 uniform field (isothermal) with the carried photons of
loop.c:745. The reference keeps its state in globals, so each case runs in
a process of its own.
"""
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def _steps(units, f, tick_time, seed, n, iso):
    from refpy import Step
    rng = np.random.default_rng(seed)
    steps = (Step * n)()
    nH = float(f.rho[0]) * units.H_PER_MASS
    for i, s in enumerate(steps):
        s.lambdaH = 10 ** rng.uniform(-4, 0)
        # (not isothermal: moderate steps, or the reference's check that one
        # whole step of cooling stays below ie, solve.c:137-139, traps)
        s.ie = float(f.ie[0]) * (1.0 if iso else 10 ** rng.uniform(0.0, 0.3))
        s.yeMET = 0.0
        s.yGdepHI = 10 ** rng.uniform(-6, -1) if rng.random() < 0.8 else 0.0
        s.heat = 0.0 if iso else s.yGdepHI * 1e-3 * float(f.ie[0])
        s.time = tick_time * int(rng.integers(1, 400 if iso else 40))
        s.nH = nH
        s.T = 1e4
    return steps


def _case(kind, q):
    from psphray_b200 import api, fields
    from psphray_b200.units import Units
    from refpy import EULER_LIB_PATH, Reference
    units = Units(hmf=1.0)
    iso = kind != "noniso"
    ref = Reference(api.RATES_HUI, units, isothermal=iso, threads=1, lib_path=EULER_LIB_PATH)
    w = fields.make_workload("iliev32", n_side=16, nray=16)
    f = w.field
    out = {}
    if kind in ("iso", "noniso"):
        steps = _steps(units, f, w.tick_time, 7 if iso else 8, 256, iso)
        fields_ = ["lambdaH", "ie", "yGdepHI", "heat", "time", "nH", "T", "yeMET"]
        for k in fields_:
            out[f"{kind}_in_{k}"] = np.array([getattr(s, k) for s in steps])
        ref.step_evolve(steps)
        for k in ("lambdaH", "ie", "step_remain", "refined"):
            out[f"{kind}_out_{k}"] = np.array([getattr(s, k) for s in steps])
    else:
        ref.load(f)
        ref.build_tree(8)
        rays_all, lam, ie, hits, lasthit = [], [], [], [], []
        for t in range(1, 21):
            rays = w.schedule.rays_for_tick(t)
            rays_all.append(rays)
            ref.set_rays(rays, t, w.tick_time)
            ref.trace()
            ref.deposit()
            ref.merge()
            ref.update()
            s = ref.state()
            lam.append(s["lambdaH"]); ie.append(s["ie"]); hits.append(s["hits"]); lasthit.append(s["lasthit"])
        out.update(tick_rays=np.concatenate(rays_all), tick_time=np.float64(w.tick_time), nray=np.int64(16),
                   st_lambdaH=np.array(lam), st_ie=np.array(ie), st_hits=np.array(hits),
                   st_lasthit=np.array(lasthit))
    q.put(out)


def main():
    ctx = mp.get_context("spawn")
    out = {}
    for kind in ("iso", "noniso", "ticks"):
        q = ctx.Queue()
        p = ctx.Process(target=_case, args=(kind, q))
        p.start()
        out.update(q.get(timeout=600))
        p.join()
        assert p.exitcode == 0, kind
    np.savez_compressed(os.path.join(HERE, "euler16.npz"), **out)
    print("wrote", os.path.join(HERE, "euler16.npz"), sorted(out))


if __name__ == "__main__":
    main()
