"""Writes the configured-length fixtures by running the reference's own code
(oracle/_ref/libpsphray_ref.so, built from the reference sources by
oracle/Makefile) for all 10,000 ticks (500 Myr) of the two uniform fields:

  long32.npz  32^3 uniform field, corner source of 5e48 photons/s at 13.6 eV,
              32 rays/tick, isothermal 1e4 K, one OpenMP thread.
              Every particle's x_HI (lambdaH), deposit counter and lasthit at
              ticks 100, 1000, 3000 and 10000; the full hit lists of ticks 1,
              5000 and 10000.
  long64.npz  the same at 64^3 with 1024 rays/tick, all host threads.
              Every 16th particle's x_HI, counter and lasthit at the same
              ticks; the ionised-volume radius and the radial x_HII profile
              of the whole field at each; the hit lists of ticks 1, 2, 5000
              and 10000 as per-ray counts plus SHA-256 digests of the
              canonical (ipar, d, b) arrays, with the first 16 rays in full.

Rays are the host schedule's (psphray_b200.fields.RaySchedule, Philox keyed
on the tick), generated tick by tick in order, as the tests regenerate them.
The reference's tick is loop.c:103-149 (trace, deposit, merge_pars,
update_pars; emission replaced by the schedule). Its float atomics make the
deposit order-dependent with more than one thread: that noise (~1e-7
relative per deposit) is far below the 1e-3 the tests allow in x_HII.

    make -C oracle ref REF=<reference tree>
    python tests/golden/make_golden_long.py [32|64]
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from psphray_b200 import fields  # noqa: E402
from psphray_b200.api import RATES_HUI  # noqa: E402

CHECKPOINTS = (100, 1000, 3000, 10000)
NTICKS = 10000
SAMPLE64 = 16          # every 16th particle of the 64^3 field is stored


def canonical_hits(ref, nray):
    """Hit lists of the last traced tick, each ray sorted by (d, ipar)."""
    ip, dd, bb, cnt = [], [], [], []
    for i in range(nray):
        a, d, b = ref.ray_hits(i)
        o = np.lexsort((a, d))
        ip.append(a[o]); dd.append(d[o]); bb.append(b[o]); cnt.append(len(a))
    cat = (lambda x: np.concatenate(x) if x else np.zeros(0))
    return (np.array(cnt, np.int32), cat(ip).astype(np.int64), cat(dd).astype(np.float64),
            cat(bb).astype(np.float64))


def hit_digest(ipar, d, b) -> str:
    """SHA-256 over the little-endian bytes of the canonical arrays (int64
    ipar, float64 d, float64 b, in that order)."""
    h = hashlib.sha256()
    for a, dt in ((ipar, "<i8"), (d, "<f8"), (b, "<f8")):
        h.update(np.ascontiguousarray(a, dt).tobytes())
    return h.hexdigest()


def ionised_radius_kpc(xHII, field):
    """Radius of the octant (corner source) whose volume equals the ionised
    volume sum(x_HII) * L^3 / N, in kpc."""
    u = field.units
    L = field.boxsize / u.KPC
    V = float(np.sum(xHII, dtype=np.float64)) * L ** 3 / field.n
    return (6.0 * V / np.pi) ** (1.0 / 3.0)


def radial_profile(xHII, field, nbins=66):
    """Mean x_HII in shells of 0.1 kpc around the corner (0,0,0)."""
    u = field.units
    r = np.sqrt((field.pos.astype(np.float64) ** 2).sum(1)) / u.KPC
    edges = np.linspace(0.0, 6.6, nbins + 1)
    idx = np.clip(np.digitize(r, edges) - 1, 0, nbins)
    s = np.bincount(idx, weights=xHII, minlength=nbins + 1)[:nbins]
    c = np.bincount(idx, minlength=nbins + 1)[:nbins]
    return np.where(c > 0, s / np.maximum(c, 1), np.nan)


def run(name, threads, sample, hit_ticks, full_hit_rays):
    from refpy import Reference
    w = fields.make_workload(name)
    f = w.field
    ref = Reference(RATES_HUI, f.units, threads=threads)
    ref.load(f)
    ref.build_tree(8)
    idx = np.arange(0, f.n, sample)
    out = dict(workload=np.array(name), seed=np.int64(20261203), n_side=np.int64(round(f.n ** (1 / 3))),
               nray=np.int64(w.schedule.nray), tick_time=np.float64(w.tick_time),
               checkpoints=np.array(CHECKPOINTS, np.int64), sample=np.int64(sample),
               hit_ticks=np.array(hit_ticks, np.int64))
    t0 = time.time()
    total_hits = 0
    for t in range(1, NTICKS + 1):
        rays = w.schedule.rays_for_tick(t)
        ref.set_rays(rays, t, w.tick_time)
        ref.trace()
        if t in hit_ticks:
            cnt, ip, dd, bb = canonical_hits(ref, len(rays))
            out[f"h{t}_count"] = cnt
            out[f"h{t}_digest"] = np.array(hit_digest(ip, dd, bb))
            if full_hit_rays is None:
                out[f"h{t}_ipar"] = ip.astype(np.int32)
                out[f"h{t}_d"] = dd
                out[f"h{t}_b"] = bb
            else:
                m = int(cnt[:full_hit_rays].sum())
                out[f"h{t}_ipar"] = ip[:m].astype(np.int32)
                out[f"h{t}_d"] = dd[:m]
                out[f"h{t}_b"] = bb[:m]
        ref.deposit()
        ref.merge()
        ref.update()
        if t in CHECKPOINTS:
            s = ref.state()
            x = 1.0 - s["lambdaH"]
            st = ref.stats()
            total_hits = st["hits"]
            out[f"c{t}_lambdaH"] = s["lambdaH"][idx].astype(np.float32)
            out[f"c{t}_hits"] = s["hits"][idx].astype(np.int32)
            out[f"c{t}_lasthit"] = s["lasthit"][idx].astype(np.int32)
            out[f"c{t}_radius_kpc"] = np.float64(ionised_radius_kpc(x, f))
            out[f"c{t}_profile"] = radial_profile(x, f)
            out[f"c{t}_total_hits"] = np.float64(total_hits)
            out[f"c{t}_saturated"] = np.float64(st["saturated"])
            print(f"{name}: tick {t} ({time.time() - t0:.0f} s) R_ion {out[f'c{t}_radius_kpc']:.3f} kpc, "
                  f"{total_hits:.0f} hits", flush=True)
    out["alpha_B_1e4"] = np.float64(ref.ar_get("HIIrcB", 4.0))
    out["threads"] = np.int64(threads)
    return out


def main():
    which = sys.argv[1:] or ["32", "64"]
    if "32" in which:
        out = run("iliev32", 1, 1, (1, 5000, 10000), None)
        np.savez_compressed(os.path.join(HERE, "long32.npz"), **out)
    if "64" in which:
        out = run("iliev64", os.cpu_count() or 1, SAMPLE64, (1, 2, 5000, 10000), 16)
        np.savez_compressed(os.path.join(HERE, "long64.npz"), **out)


if __name__ == "__main__":
    main()
