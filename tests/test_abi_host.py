"""The C ABI without a GPU: exported symbols, host-side tables against the
reference's own values, error codes. CPU only."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, load_golden


def declared_functions():
    src = open(os.path.join(ROOT, "include", "psg.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(psg_[a-z_0-9]+)\s*\(", src)
    return sorted(set(names))


def test_every_declared_symbol_is_exported(built):
    from psphray_b200 import api
    lib = C.CDLL(api.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_build_targets_sm100a_only():
    """Every nvcc step of the build (objects and the device link) carries
    exactly one -gencode, arch=compute_100a,code=sm_100a: SASS for sm_100a
    and no PTX that a driver could JIT for another architecture. The loaded
    code's architecture is checked on the GPU (test_gpu_path.py)."""
    from psphray_b200 import build
    arch = build.ARCH
    assert arch == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert build.NVCC_FLAGS.count("-gencode") == 1
    assert all(not f.startswith("-arch") and "compute_" not in f.split("code=")[-1]
               for f in build.NVCC_FLAGS if "code=" in f)


def test_tables_match_reference(phys):
    g = load_golden("tables.npz")
    for col in ["HIci", "HIIrcA", "HIIrcB", "HIIrccA", "HIIrccB", "HIcic", "HIcec", "Brem", "Compton"]:
        got = np.array([phys.ar_get(col, x) for x in g["logT"]])
        assert np.array_equal(got, g["ar_" + col]), col
    got = np.array([phys.sph_depth(x) for x in g["r_h"]])
    assert np.array_equal(got, g["sph_depth"])
    got = np.array([phys.xs_get("HI", e) for e in g["eng"]])
    ref = g["xs_HI"]
    # one unit constant differs by an ulp under the reference's -ffast-math
    m = ref != 0
    assert np.array_equal(got == 0, ref == 0)
    assert np.max(np.abs(got[m] - ref[m]) / ref[m]) < 1e-11


def test_units_match_reference(units, reference, phys):
    v = reference.units_vector()
    names = ["CM", "GRAM", "SEC", "MYR", "EV", "MPROTON", "BOLTZMANN", "H_PER_MASS", "HE_PER_MASS",
             "HI_ENERGY", "MPROTON_OVER_BOLTZMANN", "BOLTZMANN_OVER_MPROTON", "ERG", "KPC", "HEI_ENERGY",
             "HEII_ENERGY"]
    for n, x in zip(names, v):
        assert abs(phys.unit(n) - x) <= 4e-16 * abs(x), n


def test_io_errors(built, units, tmp_path):
    from psphray_b200 import api
    with pytest.raises(api.PsgError) as e:
        api.Physics(units, rates_path=str(tmp_path / "missing.txt"))
    assert e.value.code == -5
    bad = tmp_path / "short.txt"
    bad.write_text("# header only\n 0.0 9.0 2251 4.0E-03\n")
    with pytest.raises(api.PsgError) as e:
        api.Physics(units, rates_path=str(bad))
    assert e.value.code == -5
    with pytest.raises(api.PsgError) as e:
        api.Physics(units, kernel_path=str(tmp_path / "nokernel"))
    assert e.value.code == -5


def test_no_cpu_fallback(built):
    """Without a usable GPU the context cannot be created: there is no CPU
    path behind the ABI."""
    import torch
    from psphray_b200 import api
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(api.PsgError) as e:
        api.Context(0)
    assert e.value.code == -2


def test_ray_schedule_bookkeeping():
    """emit_rays() bookkeeping (loop.c:305-321, sources.c:67-78): each source's
    photons since its last emission are split evenly over its rays, so every
    tick carries L*tick_time in total once all sources have emitted."""
    from psphray_b200 import fields
    w = fields.make_workload("lognormal128", n_side=8, nray=256, seed=3)
    s = w.schedule
    L = sum(src.ngamma_dot for src in s.sources)
    total = 0.0
    for t in range(1, 6):
        rays = s.rays_for_tick(t)
        total += rays["Nph"].sum()
        assert np.all(rays["length"] == 2 * w.field.boxsize)
        n = np.sqrt((rays["dir"].astype(np.float64) ** 2).sum(1))
        assert np.all(np.abs(n - 1) < 1e-6)
    pending = sum(src.ngamma_dot * (5 - src.lastemit) * s.tick_time for src in s.sources)
    assert abs(total + pending - L * 5 * s.tick_time) < 1e-9 * L * 5 * s.tick_time


def test_fields_are_seeded():
    from psphray_b200 import fields
    a = fields.make_workload("iliev32", n_side=8, nray=4, seed=1)
    b = fields.make_workload("iliev32", n_side=8, nray=4, seed=1)
    assert np.array_equal(a.field.pos, b.field.pos) and np.array_equal(a.field.sml, b.field.sml)
    assert np.array_equal(a.schedule.rays_for_tick(3), b.schedule.rays_for_tick(3))
