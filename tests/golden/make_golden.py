"""Writes the golden fixtures under tests/golden/ by running the reference's
own code (oracle/_ref/libpsphray_ref.so, built from the reference sources by
oracle/Makefile) on small seeded cases:

  uniform16.npz   16^3 uniform field, 16 rays/tick: octree leaves, hit lists
                  of ticks 1-3, particle state after each of 40 ticks (LSODA)
  lognormal16.npz 16^3 log-normal field, 16 sources, 64 rays/tick:
                  octree leaves and the hit lists of one tick
  edges.npz       hand-made rays (axis-aligned, signed zeros, outside or on
                  the box, zero length), flagged-invalid and out-of-box
                  particles: hit lists
  tables.npz      ar_get / xs_get / sph_depth samples

    python tests/golden/make_golden.py

Run with one OpenMP thread: the reference's float atomics make the deposit
order-dependent with more.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from psphray_b200 import fields  # noqa: E402
from psphray_b200.api import RATES_HUI  # noqa: E402
from psphray_b200.units import Units  # noqa: E402


def leaves(t, n):
    """Canonical leaf description: for each particle the smallest index in its
    leaf (-1 if not in the tree) and, per non-empty leaf (keyed by that
    index), its box; plus the sorted boxes of empty leaves."""
    leaf_of = np.full(n, -1, np.int64)
    boxes = {}
    empty = []
    for c in range(len(t["head"])):
        if t["first_child"][c] != -1:
            continue
        ps = []
        p = t["head"][c]
        while p != -1:
            ps.append(int(p))
            p = t["next"][p]
        if ps:
            k = min(ps)
            leaf_of[ps] = k
            boxes[k] = np.concatenate([t["bot"][c], t["top"][c]])
        else:
            empty.append(np.concatenate([t["bot"][c], t["top"][c]]))
    keys = np.array(sorted(boxes), np.int64)
    lbox = np.array([boxes[k] for k in keys], np.float32).reshape(-1, 6)
    ebox = np.array(sorted(map(tuple, empty)), np.float32).reshape(-1, 6)
    return leaf_of, keys, lbox, ebox


def canonical_hits(ref, nray):
    ip, dd, bb, off = [], [], [], [0]
    for i in range(nray):
        a, d, b = ref.ray_hits(i)
        o = np.lexsort((a, d))
        ip.append(a[o]); dd.append(d[o]); bb.append(b[o])
        off.append(off[-1] + len(a))
    cat = (lambda x: np.concatenate(x) if x else np.zeros(0))
    return np.array(off, np.int64), cat(ip).astype(np.int64), cat(dd), cat(bb)


def field_arrays(f):
    return dict(pos=f.pos, mass=f.mass, sml=f.sml, rho=f.rho, ie=f.ie, xHI=f.xHI, ye=f.ye,
                boxsize=np.float64(f.boxsize))


def edge_rays(box, pos):
    """Rays that exercise the corner cases of the segment/box and line tests."""
    b = np.float32(box)
    c = np.float32(0.5) * b
    R = []

    def add(s, d, length):
        r = np.zeros(1, fields.RAY_DTYPE)[0]
        r["s"] = np.asarray(s, np.float32)
        d = np.asarray(d, np.float64)
        nrm = np.sqrt((d * d).sum())
        r["dir"] = (d / nrm if nrm > 0 else d).astype(np.float32)
        r["Nph"] = 1e58
        r["freq"] = 0.0
        r["length"] = length
        R.append(r)

    L = 2 * box
    for ax in range(3):
        for sgn in (1.0, -1.0):
            d = [0.0, 0.0, 0.0]
            d[ax] = sgn
            add([c, c, c], d, L)                         # from the centre, along an axis
            add([0, 0, 0], d, L)                         # from a corner
    add([c, c, c], [-0.0, 1.0, -0.0], L)                 # signed zeros
    add([c, c, c], [1.0, 1.0, 1.0], L)
    add([c, c, c], [-1.0, -1.0, -1.0], L)
    add([-b, c, c], [1.0, 0.0, 0.0], 3 * box)            # from outside, crossing
    add([-b, c, c], [-1.0, 0.0, 0.0], 3 * box)           # from outside, away
    add([2 * b, 2 * b, 2 * b], [-1.0, -1.0, -1.0], 4 * box)
    add([b, b, b], [1.0, 0.3, 0.2], L)                   # from the far corner, outward
    add([c, c, c], [0.3, -0.5, 0.8], 0.0)                # zero length
    add([c, c, c], [0.3, -0.5, 0.8], 1e-3 * box)         # very short
    add(pos[0], [0.2, 0.9, -0.1], L)                     # starting on a particle
    add(pos[1], pos[2] - pos[1], L)                      # through another particle's centre
    add([c, c, 0.0], [0.0, 0.0, 1.0], L)                 # on the box face
    return np.array(R, fields.RAY_DTYPE)


def main():
    from refpy import Reference
    units = Units(hmf=1.0)
    ref = Reference(RATES_HUI, units, threads=1)

    # ---- tables
    lt = np.linspace(-0.5, 9.5, 1001)
    ar = {c: np.array([ref.ar_get(c, x) for x in lt]) for c in
          ["HIci", "HIIrcA", "HIIrcB", "HIIrccA", "HIIrccB", "HIcic", "HIcec", "Brem", "Compton"]}
    eng = np.concatenate([np.linspace(13.0, 30.0, 500), np.geomspace(30.0, 2000.0, 500)]) * units.EV
    xs = np.array([ref.xs_get("XS_HI", e) for e in eng])
    rh = np.linspace(-0.05, 1.05, 4001)
    sd = np.array([ref.sph_depth(x) for x in rh])
    np.savez_compressed(os.path.join(HERE, "tables.npz"), logT=lt, eng=eng, xs_HI=xs, r_h=rh,
                        sph_depth=sd, **{"ar_" + k: v for k, v in ar.items()})

    # ---- uniform field, isothermal, LSODA state over 40 ticks
    w = fields.make_workload("iliev32", n_side=16, nray=16)
    f = w.field
    ref.load(f)
    ref.build_tree(8)
    leaf_of, lkeys, lbox, ebox = leaves(ref.tree(), f.n)
    out = dict(field_arrays(f), leaf_of=leaf_of, leaf_keys=lkeys, leaf_box=lbox, empty_box=ebox,
               tick_time=np.float64(w.tick_time))
    rays_all, states = [], []
    for t in range(1, 41):
        rays = w.schedule.rays_for_tick(t)
        rays_all.append(rays)
        ref.set_rays(rays, t, w.tick_time)
        ref.trace()
        if t <= 3:
            off, ip, dd, bb = canonical_hits(ref, len(rays))
            out.update({f"t{t}_off": off, f"t{t}_ipar": ip, f"t{t}_d": dd, f"t{t}_b": bb})
        ref.deposit()
        if t <= 3:
            out[f"t{t}_yGdepHI"] = ref.state()["yGdepHI"]
        ref.merge()
        if t <= 3:
            out[f"t{t}_active"] = np.sort(ref.active())
        ref.update()
        s = ref.state()
        states.append((s["lambdaH"], s["ie"], s["hits"], s["lasthit"]))
    out["rays"] = np.concatenate(rays_all)
    out["nray"] = np.int64(16)
    out["st_lambdaH"] = np.array([s[0] for s in states])
    out["st_ie"] = np.array([s[1] for s in states])
    out["st_hits"] = np.array([s[2] for s in states])
    out["st_lasthit"] = np.array([s[3] for s in states])
    np.savez_compressed(os.path.join(HERE, "uniform16.npz"), **out)

    # ---- edge cases on the same field, with flagged and out-of-box particles
    f2 = fields.make_workload("iliev32", n_side=16, nray=16).field
    f2.pos = f2.pos.copy()
    f2.pos[5] = [f2.boxsize * 1.5, 0.1, 0.1]              # outside the root: skipped
    f2.pos[6] = [np.float32(f2.boxsize), 0.2, 0.2]         # on the top face: outside (half-open)
    f2.pos[7] = [0.0, 0.0, 0.0]                            # on the bottom corner: inside
    flag = np.zeros(f2.n, np.int8)
    flag[[11, 12, 13]] = 1                                 # PF_INVALID
    # flags go through the particle loader
    keep = [np.ascontiguousarray(a) for a in (f2.pos, f2.mass, f2.sml, f2.rho, f2.ie, f2.xHI, f2.ye)]
    ref.lib.ref_load_particles(f2.n, *[a.ctypes.data for a in keep], flag.ctypes.data, f2.boxsize)
    ref.build_tree(8)
    leaf_of, lkeys, lbox, ebox = leaves(ref.tree(), f2.n)
    rays = edge_rays(f2.boxsize, f2.pos)
    ref.set_rays(rays, 1, w.tick_time)
    ref.trace()
    off, ip, dd, bb = canonical_hits(ref, len(rays))
    np.savez_compressed(os.path.join(HERE, "edges.npz"), **field_arrays(f2), flag=flag, rays=rays,
                        off=off, ipar=ip, d=dd, b=bb, leaf_of=leaf_of, leaf_keys=lkeys, leaf_box=lbox,
                        empty_box=ebox)

    # ---- log-normal field, several sources
    w3 = fields.make_workload("lognormal128", n_side=16, nray=64)
    f3 = w3.field
    ref.load(f3)
    ref.build_tree(8)
    leaf_of, lkeys, lbox, ebox = leaves(ref.tree(), f3.n)
    rays = w3.schedule.rays_for_tick(1)
    ref.set_rays(rays, 1, w3.tick_time)
    ref.trace()
    off, ip, dd, bb = canonical_hits(ref, len(rays))
    np.savez_compressed(os.path.join(HERE, "lognormal16.npz"), **field_arrays(f3), rays=rays, off=off,
                        ipar=ip, d=dd, b=bb, leaf_of=leaf_of, leaf_keys=lkeys, leaf_box=lbox, empty_box=ebox)

    print("wrote", sorted(x for x in os.listdir(HERE) if x.endswith(".npz")))


if __name__ == "__main__":
    main()
