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


def _snapshot(tmp_path):
    from psphray_b200 import api, fields
    w = fields.make_workload("iliev32", n_side=8, nray=16, seed=4)
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
