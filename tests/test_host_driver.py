"""psg_run, the C host driver over the library's C ABI (one epoch of
run_epoch(): snapshot in, tables, tree, device-emitted ticks, snapshot out):
built as plain C11 against include/psg.h; its argument and file checks; and,
on a machine without a GPU, the host side up to psg_create() -- the
snapshot read and the tables built -- and a clean library error there."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUN = os.path.join(ROOT, "psphray_b200", "psg_run")


def _run(*args):
    return subprocess.run([RUN, *map(str, args)], capture_output=True, text=True, timeout=120)


def _snapshot(tmp_path, n_side=8):
    from psphray_b200 import api, fields
    w = fields.make_workload("iliev32", n_side=n_side, nray=16, seed=4)
    f = w.field
    path = str(tmp_path / "in.psphray")
    api.write_snapshot(path, f.n, {"pos": f.pos, "mass": f.mass, "sml": f.sml, "rho": f.rho, "ie": f.ie,
                                   "xHI": f.xHI, "ye": f.ye, "id": np.arange(f.n, dtype=np.int64)},
                       src_pos=np.zeros((1, 3), np.float32), ngammas=np.array([w.schedule.sources[0].ngamma_dot]),
                       boxsize=f.boxsize, h=0.72, time=1.0)
    return path


def test_driver_builds_and_checks_arguments(built, tmp_path):
    assert os.access(RUN, os.X_OK)
    r = _run()
    assert r.returncode == 1 and "usage: psg_run" in r.stderr
    from psphray_b200.api import KERNEL_AKLINE, RATES_HUI
    r = _run(tmp_path / "missing", RATES_HUI, KERNEL_AKLINE, 4, 16, 1.0, tmp_path / "out")
    assert r.returncode == 2 and "not a psphray-format file" in r.stderr
    snap = _snapshot(tmp_path)
    r = _run(snap, RATES_HUI, KERNEL_AKLINE, 0, 16, 1.0, tmp_path / "out")
    assert r.returncode == 1
    r = _run(snap, RATES_HUI, KERNEL_AKLINE, 4, 16, 1.0, tmp_path / "out", "--blackbody", "-1")
    assert r.returncode == 1
    r = _run(snap, tmp_path / "no-rates", KERNEL_AKLINE, 4, 16, 1.0, tmp_path / "out")
    assert r.returncode == 2 and "cannot build the tables" in r.stderr


def test_driver_host_side_without_gpu(built, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the driver would run the ticks")
    from psphray_b200.api import KERNEL_AKLINE, RATES_HUI
    snap = _snapshot(tmp_path)
    r = _run(snap, RATES_HUI, KERNEL_AKLINE, 4, 16, 1.0, tmp_path / "out", "--isothermal", "--batch", "2")
    assert r.returncode == 3, r.stderr
    assert "psg_create" in r.stderr
    assert not os.path.exists(tmp_path / "out")


@pytest.mark.gpu
def test_driver_epoch_matches_binding(built, tmp_path):
    """16 ticks of 64 device-emitted rays on a 16^3 field, once through the
    driver and once through the Python binding with the same source, seed
    and tick time: hit counters and lasthit equal, the output's xHI the
    float of lambdaH (to 1e-6: the C and Python unit constants may differ
    in the last bit)."""
    from types import SimpleNamespace
    from psphray_b200 import api, fields
    from psphray_b200.api import KERNEL_AKLINE, RATES_HUI
    snap = _snapshot(tmp_path, n_side=16)
    out = tmp_path / "out.psphray"
    seed = 77
    r = _run(snap, RATES_HUI, KERNEL_AKLINE, 16, 64, 0.8, out, "--isothermal", "--batch", "8", "--seed", seed)
    assert r.returncode == 0, r.stderr
    assert "16 ticks of 64 rays" in r.stdout
    w = fields.make_workload("iliev32", n_side=16, nray=16, seed=4)
    f = w.field
    ctx = api.Context(0)
    try:
        ctx.set_physics(api.Physics(f.units, isothermal=True))
        ctx.load(f)
        ctx.build_tree(8)
        src = SimpleNamespace(pos=(0.0, 0.0, 0.0), ngamma_dot=w.schedule.sources[0].ngamma_dot, lastemit=0)
        ctx.set_sources([src], [(np.array([13.6 * f.units.EV]), np.array([1.0]))], seed=seed)
        tick_time = 0.8 * f.units.MYR / 16
        ctx.run_ticks_emit(64, 8, 1, tick_time)
        ctx.run_ticks_emit(64, 8, 9, tick_time)
        st = ctx.state()
    finally:
        ctx.close()
    o = api.read_snapshot(str(out))
    assert (st["lasthit"] > 0).sum() > 1000
    assert np.array_equal(o["lasthit"], st["lasthit"])
    assert np.array_equal(o["hits"], st["hits"])
    assert np.max(np.abs(o["xHI"].astype(np.float64) - st["lambdaH"].astype(np.float32))) <= 1e-6


@pytest.mark.gpu
def test_driver_resume_keeps_helium(built, tmp_path):
    """An epoch with helium (--hmf 0.76, a 1e5 K blackbody reaching past
    the HeII edge) writes its output; a second epoch starts from that file.
    With --resume the particles the second epoch does not hit keep the
    file's xHeI and xHeII exactly; without it the load derives them from ye
    (psystem.c:340-358), which puts every helium electron on HeII first and
    so moves the particles that held HeIII."""
    from psphray_b200 import api
    from psphray_b200.api import KERNEL_AKLINE, RATES_HUI
    snap = _snapshot(tmp_path, n_side=16)
    a = tmp_path / "a.psphray"
    r = _run(snap, RATES_HUI, KERNEL_AKLINE, 40, 256, 40.0, a, "--hmf", "0.76", "--blackbody", "1e5")
    assert r.returncode == 0, r.stderr
    A = api.read_snapshot(str(a))
    heIII = 1.0 - A["xHeI"].astype(np.float64) - A["xHeII"]
    assert (heIII > 1e-3).sum() > 10
    outs = {}
    for tag, extra in (("resume", ["--resume"]), ("derive", [])):
        b = tmp_path / f"b_{tag}.psphray"
        r = _run(a, RATES_HUI, KERNEL_AKLINE, 1, 4, 0.01, b, "--hmf", "0.76", *extra)
        assert r.returncode == 0, r.stderr
        outs[tag] = api.read_snapshot(str(b))
    B = outs["resume"]
    cold = B["lasthit"] == 0
    assert cold.sum() > 0.5 * len(cold)
    assert np.array_equal(B["xHeI"][cold], A["xHeI"][cold])
    assert np.array_equal(B["xHeII"][cold], A["xHeII"][cold])
    D = outs["derive"]
    cold_d = D["lasthit"] == 0
    moved = cold_d & (heIII > 1e-3)
    assert moved.sum() > 0
    assert np.any(D["xHeII"][moved] != A["xHeII"][moved])
