"""Shared fixtures. GPU tests are marked ``gpu``; everything else runs on CPU.

The checker for every GPU test is the C restatement in oracle/ (built here
from source if missing); the restatement itself is pinned by the golden
fixtures under tests/golden/, which come from the reference's own code, and
by live comparisons with that code when oracle/_ref/libpsphray_ref.so exists.
"""
from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_oracle():
    lib = os.path.join(ROOT, "oracle", "_ref", "libpsg_oracle.so")
    src = os.path.join(ROOT, "oracle", "psg_oracle.c")
    if not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True,
                       capture_output=True)


def _ensure_lib():
    from psphray_b200 import build
    build.build()


@pytest.fixture(scope="session", autouse=True)
def built():
    _ensure_oracle()
    _ensure_lib()


def load_golden(name: str) -> dict:
    with np.load(os.path.join(GOLDEN, name)) as z:
        return {k: z[k] for k in z.files}


def golden_field(g: dict):
    from psphray_b200.fields import Field
    from psphray_b200.units import Units
    return Field(pos=g["pos"], mass=g["mass"], sml=g["sml"], rho=g["rho"], ie=g["ie"], xHI=g["xHI"],
                 ye=g["ye"], boxsize=float(g["boxsize"]), units=Units(hmf=1.0))


@pytest.fixture(scope="session")
def units():
    from psphray_b200.units import Units
    return Units(hmf=1.0)


@pytest.fixture(scope="session")
def phys(units, built):
    from psphray_b200 import api
    return api.Physics(units)


@pytest.fixture(scope="session")
def phys_noniso(units, built):
    from psphray_b200 import api
    return api.Physics(units, isothermal=False)


@pytest.fixture(scope="session")
def reference(units):
    """The reference's own code; skipped where it was not built (it needs the
    reference sources at build time)."""
    from refpy import LIB_PATH, Reference
    if not os.path.exists(LIB_PATH):
        pytest.skip("oracle/_ref/libpsphray_ref.so not built here")
    from psphray_b200.api import RATES_HUI
    return Reference(RATES_HUI, units, threads=1)


@pytest.fixture(scope="session")
def gpu_ctx(built):
    from psphray_b200 import api
    try:
        ctx = api.Context(0)
    except api.PsgError as e:
        pytest.fail(f"no usable GPU for a gpu-marked test: {e}")
    yield ctx
    ctx.close()


def leaf_sets_from_oracle(t, n):
    """Canonical leaves of a pointer octree (reference or restatement)."""
    leaf_of = np.full(n, -1, np.int64)
    boxes, empty = {}, []
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
    return (leaf_of, keys, np.array([boxes[k] for k in keys], np.float32).reshape(-1, 6),
            np.array(sorted(map(tuple, empty)), np.float32).reshape(-1, 6))


def leaf_sets_from_gpu(t, n):
    """Canonical leaves of the depth-first device tree."""
    skip, pstart, order = t["skip"], t["pstart"], t["order"]
    leaf_of = np.full(n, -1, np.int64)
    boxes, empty = {}, []
    for i in range(t["ncells"]):
        if skip[i] != i + 1:
            continue
        ps = order[pstart[i]:pstart[i + 1]]
        box = np.concatenate([t["bot"][i], t["top"][i]])
        if len(ps):
            k = int(ps.min())
            leaf_of[ps] = k
            boxes[k] = box
        else:
            empty.append(box)
    keys = np.array(sorted(boxes), np.int64)
    return (leaf_of, keys, np.array([boxes[k] for k in keys], np.float32).reshape(-1, 6),
            np.array(sorted(map(tuple, empty)), np.float32).reshape(-1, 6))
