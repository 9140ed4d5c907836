"""Golden ticks of a run that is not isothermal, hydrogen only and on the
spot, from the reference's own code with its LSODA solver
(oracle/_ref/libpsphray_ref.so, `make -C oracle ref REF=<psphray tree>`):

    python tests/golden/make_golden_noniso.py

writes tests/golden/noniso16.npz: the 16^3 uniform field heated by a corner
source of 5e48 photons/s with a 1e5 K blackbody in 4 lines over 1-1.5 Ry
(every absorption heats), 256 rays per tick of the host schedule
(psphray_b200.fields), 60 ticks of trace(), deposit(), merge_pars() and
update_pars() (loop.c:131-147; step_evolve_lsoda() solve.c:170-224
integrating x_HI and the internal energy), the particle state after ticks
1, 10, 30 and 60. The gas warms to ~5e4 K at the front. The reference's
right-hand side traps (solve.c:137-139) where one whole step of cooling
would exceed the internal energy: harder spectra (lines up to 4 or 10 Ry)
heat the front particles into that regime and trap, so the spectrum is
kept soft. One OpenMP thread (its float atomics make the deposit
order-dependent with more).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

NTICK = 60
CHECK = (1, 10, 30, 60)


def workload():
    from psphray_b200 import fields
    w = fields.make_workload("iliev32", n_side=16, nray=256, seed=21)
    u = w.field.units
    e, wt = fields.blackbody_bins(u, T=1e5, nbins=4, emin_ry=1.0, emax_ry=1.5)
    w.schedule.energies, w.schedule.eweights = e, wt
    w.schedule.sources[0].ngamma_dot = 5e48 / u.SEC
    return w


def main():
    from refpy import Reference
    from psphray_b200.api import RATES_HUI
    w = workload()
    f = w.field
    ref = Reference(RATES_HUI, f.units, isothermal=False, threads=1)
    ref.load(f)
    ref.build_tree(8)
    out = {"tick_time": np.float64(w.tick_time), "nray": np.int64(w.schedule.nray),
           "checkpoints": np.array(CHECK, np.int64)}
    rays = []
    for t in range(1, NTICK + 1):
        r = w.schedule.rays_for_tick(t)
        rays.append(r)
        ref.tick(r, t, w.tick_time)
        if t in CHECK:
            s = ref.state()
            out[f"c{t}_lambdaH"] = s["lambdaH"]
            out[f"c{t}_ie"] = s["ie"]
            out[f"c{t}_hits"] = s["hits"]
            out[f"c{t}_lasthit"] = s["lasthit"]
    out["rays"] = np.concatenate(rays)
    np.savez_compressed(os.path.join(HERE, "noniso16.npz"), **out)
    print("wrote noniso16.npz")


if __name__ == "__main__":
    main()
