"""Golden vectors for runs not on the spot (psphray.onTheSpot = false), from
the reference's own code (oracle/_ref/libpsphray_ref.so, `make -C oracle
ref`).

    python tests/golden/make_golden_recomb.py

writes tests/golden/recomb16.npz:

- Step records before and after step_evolve() (solve.c:170-224, LSODA),
  isothermal and not, with case-A recombination and the recombination
  photons yGrecHII integrated (solve.c:83-86);
- ticks of the 16^3 uniform field, isothermal: per tick the state before
  (lambdaH, ie, lasthit, hits, yGrecHII and the tick each particle was last
  hit by a source ray), the tick's recombination rays (made by the oracle's
  restatement of the device's emission, oracle/recomb.py, from that state:
  the reference's GSL draws have no device counterpart) and the state after
  the reference's trace(), deposit(), merge_pars() and update_pars() ran
  the tick's source rays and those recombination rays. Once with nrec draws
  per tick, once in threshold mode (nrec < 0).

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

NTICK = 10
NREC = 24
SEED = 7
THRESHOLD = 2e-4


def _steps(f, tick_time, seed, n, iso, units):
    from refpy import Step
    rng = np.random.default_rng(seed)
    steps = (Step * n)()
    nH = float(f.rho[0]) * units.H_PER_MASS
    for s in steps:
        s.lambdaH = 10 ** rng.uniform(-4, 0)
        s.ie = float(f.ie[0]) * (1.0 if iso else 10 ** rng.uniform(0.0, 0.3))
        s.yeMET = 0.0
        s.yGdepHI = 10 ** rng.uniform(-6, -1) if rng.random() < 0.8 else 0.0
        s.heat = 0.0 if iso else s.yGdepHI * 1e-3 * float(f.ie[0])
        s.time = tick_time * int(rng.integers(1, 400 if iso else 40))
        s.nH = nH
        s.T = 1e4
        s.yGrecHII = rng.uniform(0.0, 0.5)
    return steps


def consts_of(phys):
    return {k: phys.unit(k) for k in ("HI_ENERGY", "BOLTZMANN", "H_PER_MASS", "MPROTON_OVER_BOLTZMANN",
                                      "hmf", "hemf")}


def _case(kind, q):
    import recomb
    from psphray_b200 import api, fields
    from psphray_b200.units import Units
    from refpy import Reference
    units = Units(hmf=1.0)
    iso = kind != "noniso"
    ref = Reference(api.RATES_HUI, units, isothermal=iso, on_the_spot=False, threads=1)
    w = fields.make_workload("iliev32", n_side=16, nray=16)
    f = w.field
    out = {}
    if kind in ("iso", "noniso"):
        steps = _steps(f, w.tick_time, 11 if iso else 12, 256, iso, units)
        names = ["lambdaH", "ie", "yGdepHI", "heat", "time", "nH", "T", "yeMET", "yGrecHII"]
        for k in names:
            out[f"{kind}_in_{k}"] = np.array([getattr(s, k) for s in steps])
        ref.step_evolve(steps)
        for k in ("lambdaH", "ie", "yGrecHII"):
            out[f"{kind}_out_{k}"] = np.array([getattr(s, k) for s in steps])
    else:
        nrec = NREC if kind == "ticks" else -1
        phys = api.Physics(units, isothermal=True, on_the_spot=False)
        c = consts_of(phys)
        lte = recomb.lte_table(c["HI_ENERGY"], c["BOLTZMANN"], lambda e: phys.xs_get("HI", e))
        ref.load(f)
        ref.build_tree(8)
        pos = np.asarray(f.pos, np.float32).reshape(-1, 3)
        mass = np.asarray(f.mass, np.float32)
        mark = np.full(f.n, -1, np.int32)
        rec = {k: [] for k in ("b_lambdaH", "b_ie", "b_lasthit", "b_hits", "b_ygrec", "b_mark", "a_lambdaH", "a_ie",
                               "a_lasthit", "a_hits", "a_ygrec", "a_mark", "src_rays", "rec_rays", "rec_ipar")}
        R = w.schedule.nray
        for t in range(1, NTICK + 1):
            s = ref.state()
            yg = ref.ygrec()
            for k, v in (("lambdaH", s["lambdaH"]), ("ie", s["ie"]), ("lasthit", s["lasthit"]), ("hits", s["hits"]),
                         ("ygrec", yg), ("mark", mark.copy())):
                rec["b_" + k].append(v)
            src = w.schedule.rays_for_tick(t)
            rays_rec, em, yg2 = recomb.emit(yg, s["lambdaH"], mark, pos, mass, s["ie"], t, nrec, SEED, f.boxsize, c,
                                            lte=lte, threshold=THRESHOLD) if t > 1 else \
                (np.zeros(0, src.dtype), np.zeros(0, np.int64), yg)
            ref.set_ygrec(yg2)
            ref.set_rays(np.concatenate([src, rays_rec]), t, w.tick_time)
            ref.trace(); ref.deposit(); ref.merge(); ref.update()
            for i in range(R + (1 if len(rays_rec) else 0)):
                mark[ref.ray_hits(i)[0]] = t
            s = ref.state()
            for k, v in (("lambdaH", s["lambdaH"]), ("ie", s["ie"]), ("lasthit", s["lasthit"]), ("hits", s["hits"]),
                         ("ygrec", ref.ygrec()), ("mark", mark.copy())):
                rec["a_" + k].append(v)
            rec["src_rays"].append(src)
            rec["rec_rays"].append(rays_rec)
            rec["rec_ipar"].append(em)
        p = kind + "_"
        for k in rec:
            if k in ("rec_rays", "rec_ipar"):
                out[p + k] = np.concatenate(rec[k])
                out[p + k + "_n"] = np.array([len(x) for x in rec[k]], np.int64)
            else:
                out[p + k] = np.stack(rec[k])
        out[p + "nrec"] = np.int64(nrec)
    out["tick_time"] = np.float64(w.tick_time)
    q.put(out)


def main():
    ctx = mp.get_context("spawn")
    out = {"seed": np.int64(SEED), "threshold": np.float64(THRESHOLD)}
    for kind in ("iso", "noniso", "ticks", "ticksthr"):
        q = ctx.Queue()
        p = ctx.Process(target=_case, args=(kind, q))
        p.start()
        out.update(q.get(timeout=900))
        p.join()
        assert p.exitcode == 0, kind
    np.savez_compressed(os.path.join(HERE, "recomb16.npz"), **out)
    print("wrote", os.path.join(HERE, "recomb16.npz"), sorted(out))


if __name__ == "__main__":
    main()
