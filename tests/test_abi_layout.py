"""The Python binding's mirrors of include/psg.h's structs (ctypes structures
and numpy dtypes in psphray_b200/api.py and fields.py) against the C
compiler's own layout: a small C program, generated from the mirrors'
field names, prints sizeof and offsetof of every field; a field renamed,
added or moved on one side only fails here, without a GPU."""
import ctypes as C
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _mirrors():
    from psphray_b200 import api, fields
    structs = [
        (api.UnitParams, "psg_unit_params"), (api.CUnits, "psg_units"), (api.RateTable, "psg_rate_table"),
        (api.XsTable, "psg_xs_table"), (api.Flags, "psg_flags"), (api.Particles, "psg_particles"),
        (api.TreeInfo, "psg_tree_info"), (api.CSource, "psg_source"), (api.CSnapshot, "psg_snapshot"),
        (api.Tune, "psg_tune"), (api.CSpectrum, "psg_spectrum"), (api.TickStats, "psg_tick_stats"),
    ]
    out = []
    for cls, cname in structs:
        out.append((cname, C.sizeof(cls), [(f[0], getattr(cls, f[0]).offset) for f in cls._fields_]))
    for dt, cname in ((fields.RAY_DTYPE, "psg_ray"), (api.XTYPE_DTYPE, "psg_xtype"), (api.STEP_DTYPE, "psg_step")):
        out.append((cname, dt.itemsize, [(n, dt.fields[n][1]) for n in dt.names if not n.startswith("_")]))
    return out


def test_binding_mirrors_match_the_header(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    mirrors = _mirrors()
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "psg.h"', "int main(void) {"]
    for cname, _, flds in mirrors:
        lines.append(f'\tprintf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f, _ in flds:
            lines.append(f'\tprintf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["\treturn 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True,
                   capture_output=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, f, v = line.split()
        got[(cname, f)] = int(v)
    for cname, size, flds in mirrors:
        assert got[(cname, "sizeof")] == size, cname
        for f, off in flds:
            assert got[(cname, f)] == off, (cname, f)
