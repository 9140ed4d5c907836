"""psystem_write_output() from device state (psg_write_output) and a run
resumed from that file: the file holds the state the context reports, and
the resumed run follows the uninterrupted one to the float precision the
format stores (xHI, ie as float)."""
import numpy as np
import pytest

from conftest import golden_field, load_golden

pytestmark = pytest.mark.gpu

CONSTS = dict(time=0.1, redshift=9.0, OmegaM=0.26, OmegaL=0.74, OmegaB=0.044, h=0.72)


def _ctx(field, phys):
    from psphray_b200 import api
    c = api.Context(0)
    c.set_physics(phys)
    c.load(field)
    c.build_tree(8)
    return c


def test_output_and_resume(phys, tmp_path):
    from psphray_b200 import api
    from psphray_b200.fields import Field
    g = load_golden("uniform16.npz")
    f = golden_field(g)
    R, tt = int(g["nray"]), float(g["tick_time"])
    rays = g["rays"]
    a = _ctx(f, phys)
    b = None
    try:
        a.run_ticks(rays[:8 * R], R, 8, 1, tt)
        path = str(tmp_path / "output_000")
        a.write_output(path, boxsize=f.boxsize, **CONSTS)
        r = api.read_snapshot(path)
        st = a.state()
        assert r["ngas"] == f.n and r["boxsize"] == f.boxsize and r["redshift"] == CONSTS["redshift"]
        assert np.array_equal(r["pos"], np.asarray(f.pos, np.float32).reshape(-1, 3))
        for k in ("mass", "sml", "rho"):
            assert np.array_equal(r[k], np.asarray(getattr(f, k), np.float32)), k
        assert np.array_equal(r["xHI"], st["lambdaH"].astype(np.float32))
        assert np.array_equal(r["ie"], st["ie"])
        assert np.array_equal(r["hits"], st["hits"]) and np.array_equal(r["lasthit"], st["lasthit"])
        assert np.array_equal(r["id"], np.arange(f.n))
        # resume: a new context from the file continues as the original does
        f2 = Field(pos=r["pos"], mass=r["mass"], sml=r["sml"], rho=r["rho"], ie=r["ie"], xHI=r["xHI"], ye=r["ye"],
                   boxsize=f.boxsize, units=f.units)
        b = _ctx(f2, phys)
        b.set_state(lasthit=r["lasthit"])
        b.set_hits(r["hits"])
        a.run_ticks(rays[8 * R:16 * R], R, 8, 9, tt)
        b.run_ticks(rays[8 * R:16 * R], R, 8, 9, tt)
        sa, sb = a.state(), b.state()
        assert np.array_equal(sa["hits"], sb["hits"]) and np.array_equal(sa["lasthit"], sb["lasthit"])
        # the file stores x_HI in float: the runs differ by about a float ulp
        assert np.max(np.abs(sa["lambdaH"] - sb["lambdaH"])) < 1e-6
    finally:
        a.close()
        if b is not None:
            b.close()
