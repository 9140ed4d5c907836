"""Python binding of libpsg (include/psg.h) through ctypes.

Mirrors the reference's entry points on the hot path: ``rt_switch_epoch``
(``Context.build_tree``), ``rt_trace`` (``Context.rt_trace``), the tick
phases of ``run_epoch`` (``Context.run_ticks``), ``step_evolve``
(``Context.step_evolve``) and the table getters ``ar_get`` / ``xs_get`` /
``sph_depth``. Errors raise ``PsgError`` carrying the library's status code
and message instead of trapping.

There is no CPU fallback: without the built library or a GPU the calls fail.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .fields import RAY_DTYPE, Field

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpsg.so")
DATA = os.path.join(HERE, "data")
RATES_HUI = os.path.join(DATA, "atomic_rates_Hui.txt")
KERNEL_AKLINE = os.path.join(DATA, "kernel.akline")

PSG_OK = 0
ERRORS = {-1: "PSG_E_INVAL", -2: "PSG_E_CUDA", -3: "PSG_E_NOMEM", -4: "PSG_E_OVERFLOW",
          -5: "PSG_E_IO", -6: "PSG_E_DEVICE"}
AR_COLS = ["HIci", "HIIrcA", "HIIrcB", "HIIrccA", "HIIrccB", "HIcic", "HIcec", "Brem", "Compton",
           "HeIci", "HeIIci", "HeIIrcA", "HeIIrcB", "HeIIIrcA", "HeIIIrcB"]
XS_SPECIES = ["HI", "HeI", "HeII"]


class PsgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class UnitParams(C.Structure):
    _fields_ = [("h", C.c_double), ("hmf", C.c_double), ("length_cmh", C.c_double),
                ("mass_gramh", C.c_double), ("time_sh", C.c_double)]


_UNIT_NAMES = ["CM", "GRAM", "SEC", "M", "KM", "KPC", "YR", "MYR", "KG", "MSUN", "MPROTON", "KELVIN",
               "BOLTZMANN", "J", "EV", "ERG", "RY_ENG", "H_PER_MASS", "HE_PER_MASS", "HI_ENERGY",
               "HEI_ENERGY", "HEII_ENERGY", "MPROTON_OVER_BOLTZMANN", "BOLTZMANN_OVER_MPROTON",
               "hmf", "hemf"]


class CUnits(C.Structure):
    _fields_ = [(n, C.c_double) for n in _UNIT_NAMES]


class RateTable(C.Structure):
    _fields_ = [("nrows", C.c_int), ("min", C.c_double), ("max", C.c_double), ("step", C.c_double),
                ("step_inv", C.c_double), ("logT", C.POINTER(C.c_double)),
                ("col", C.POINTER(C.c_double) * len(AR_COLS))]


class XsTable(C.Structure):
    _fields_ = [("nrows", C.c_int), ("min", C.c_double), ("max", C.c_double), ("step", C.c_double),
                ("step_inv", C.c_double), ("eng", C.POINTER(C.c_double)),
                ("sigma", C.POINTER(C.c_double) * 3), ("cut", C.c_double * 3)]


class Flags(C.Structure):
    _fields_ = [("isothermal", C.c_int), ("on_the_spot", C.c_int), ("h_only", C.c_int),
                ("adiabatic", C.c_int), ("euler", C.c_int), ("secondary_ionization", C.c_int)]


class Particles(C.Structure):
    _fields_ = [("n", C.c_size_t), ("pos", C.c_void_p), ("mass", C.c_void_p), ("sml", C.c_void_p),
                ("rho", C.c_void_p), ("ie", C.c_void_p), ("xHI", C.c_void_p), ("ye", C.c_void_p),
                ("flag", C.c_void_p), ("boxsize", C.c_double)]


class TreeInfo(C.Structure):
    _fields_ = [("ncells", C.c_size_t), ("nleaves", C.c_size_t), ("skipped", C.c_size_t),
                ("depth", C.c_int)]


KERNELS = ["trace_count", "trace_fill", "sort", "slots", "deposit", "update", "emit"]

SRC_PLANE, SRC_POINT = 0, 1


class CSource(C.Structure):
    _fields_ = [("type", C.c_int), ("specid", C.c_int), ("pos", C.c_double * 3), ("dir", C.c_double * 3),
                ("a", C.c_double * 3), ("b", C.c_double * 3), ("radius", C.c_double),
                ("ticks", C.c_void_p), ("ngamma_dot", C.c_void_p), ("nhist", C.c_int),
                ("lastemit", C.c_int64)]


class CSnapshot(C.Structure):
    _fields_ = [("ngas", C.c_size_t), ("nsrc", C.c_size_t)] + [
        (n, C.c_double) for n in ("time", "redshift", "boxsize", "OmegaM", "OmegaL", "OmegaB", "h")] + [
        (n, C.c_void_p) for n in ("pos", "id", "mass", "ie", "rho", "ye", "xHI", "sml", "xHeI", "xHeII",
                                  "gammaHI", "lasthit", "hits", "src_pos", "ngammas")]


SNAP_ARRAYS = {"pos": (np.float32, 3), "id": (np.int64, 1), "mass": (np.float32, 1), "ie": (np.float32, 1),
               "rho": (np.float32, 1), "ye": (np.float32, 1), "xHI": (np.float32, 1), "sml": (np.float32, 1),
               "xHeI": (np.float32, 1), "xHeII": (np.float32, 1), "gammaHI": (np.float32, 1),
               "lasthit": (np.int64, 1), "hits": (np.int32, 1)}
SNAP_CONSTS = ("time", "redshift", "boxsize", "OmegaM", "OmegaL", "OmegaB", "h")


def write_snapshot(path: str, ngas: int, arrays: dict, src_pos=None, ngammas=None, **consts):
    """psphray-format file from host arrays (missing ones written as zeros)."""
    s = CSnapshot(ngas=ngas, nsrc=0 if src_pos is None else len(src_pos))
    for k in SNAP_CONSTS:
        setattr(s, k, float(consts.get(k, 0.0)))
    keep = []
    for k, (dt, _) in SNAP_ARRAYS.items():
        if arrays.get(k) is not None:
            a = np.ascontiguousarray(arrays[k], dt)
            keep.append(a)
            setattr(s, k, a.ctypes.data)
    if src_pos is not None:
        sp = np.ascontiguousarray(src_pos, np.float32); ng = np.ascontiguousarray(ngammas, np.float64)
        keep += [sp, ng]
        s.src_pos, s.ngammas = sp.ctypes.data, ng.ctypes.data
    rc = lib().psg_snapshot_write(path.encode(), C.byref(s))
    if rc != PSG_OK:
        raise PsgError(rc, f"psg_snapshot_write({path})")


def read_snapshot(path: str) -> dict:
    """Every block of a psphray-format file: arrays and constants."""
    s = CSnapshot()
    rc = lib().psg_snapshot_read_header(path.encode(), C.byref(s))
    if rc != PSG_OK:
        raise PsgError(rc, f"psg_snapshot_read_header({path})")
    out = {k: getattr(s, k) for k in SNAP_CONSTS}
    out["ngas"], out["nsrc"] = s.ngas, s.nsrc
    for k, (dt, w) in SNAP_ARRAYS.items():
        a = np.zeros((s.ngas, w) if w > 1 else s.ngas, dt)
        out[k] = a
        setattr(s, k, a.ctypes.data)
    out["src_pos"] = np.zeros((s.nsrc, 3), np.float32)
    out["ngammas"] = np.zeros(s.nsrc, np.float64)
    s.src_pos, s.ngammas = out["src_pos"].ctypes.data, out["ngammas"].ctypes.data
    rc = lib().psg_snapshot_read(path.encode(), C.byref(s))
    if rc != PSG_OK:
        raise PsgError(rc, f"psg_snapshot_read({path})")
    return out


class Tune(C.Structure):
    """psg_tune: launch shapes that do not change results."""
    _fields_ = [("trace_warps", C.c_int), ("deposit_long", C.c_int), ("deposit_mid", C.c_int),
                ("update_minblocks", C.c_int), ("leaf_size", C.c_int), ("run_short", C.c_int),
                ("update_order", C.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class CSpectrum(C.Structure):
    _fields_ = [("eng", C.c_void_p), ("weight", C.c_void_p), ("n", C.c_int)]


class TickStats(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("hits", "saturated", "active", "lost_photons",
                                          "trace_ms", "tick_ms", "launches")] + [
        ("kernel_ms", C.c_double * len(KERNELS)), ("kernel_launches", C.c_double * len(KERNELS)),
        ("surrogate_accepted", C.c_double), ("rec_rays", C.c_double), ("rec_photons", C.c_double),
        ("host_syncs", C.c_double)]


def _stats(st: TickStats) -> dict:
    d = {k: getattr(st, k) for k, _ in TickStats._fields_[:7]}
    d["kernel_ms"] = dict(zip(KERNELS, list(st.kernel_ms)))
    d["kernel_launches"] = dict(zip(KERNELS, list(st.kernel_launches)))
    d["surrogate_accepted"] = st.surrogate_accepted
    d["rec_rays"] = st.rec_rays
    d["rec_photons"] = st.rec_photons
    d["host_syncs"] = st.host_syncs
    return d


XTYPE_DTYPE = np.dtype([("ipar", "<i8"), ("d", "<f8"), ("b", "<f8")])
STEP_DTYPE = np.dtype([(n, "<f8") for n in (
    "lambdaH", "lambdaHeI", "lambdaHeII", "ie", "yeMET", "yGdepHI", "yGdepHeI", "yGdepHeII", "heat",
    "time", "nH", "T", "yGrecHII", "yGrecHeII", "yGrecHeIII", "step_remain")]
    + [("refined", "<i4"), ("_pad", "<i4"), ("ipar", "<i8")])

_lib = None


def lib() -> C.CDLL:
    """Loads libpsg.so (built by psphray_b200.build); fails loudly if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: run `python -m psphray_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, sz, i64, dbl = C.c_void_p, C.c_size_t, C.c_int64, C.c_double
    sig = {
        "psg_units_init": ([C.POINTER(UnitParams), C.POINTER(CUnits)], C.c_int),
        "psg_rate_table_load": ([C.c_char_p, C.POINTER(CUnits), C.POINTER(RateTable)], C.c_int),
        "psg_rate_table_free": ([C.POINTER(RateTable)], None),
        "psg_ar_get": ([C.POINTER(RateTable), C.c_int, dbl], dbl),
        "psg_xs_table_build": ([C.POINTER(CUnits), C.POINTER(XsTable)], C.c_int),
        "psg_xs_table_free": ([C.POINTER(XsTable)], None),
        "psg_xs_get": ([C.POINTER(XsTable), C.c_int, dbl], dbl),
        "psg_kernel_table_load": ([C.c_char_p, vp, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "psg_sph_depth": ([vp, C.c_int, dbl], dbl),
        "psg_create": ([C.POINTER(vp), C.c_int], C.c_int),
        "psg_destroy": ([vp], None),
        "psg_last_error": ([vp], C.c_char_p),
        "psg_set_stream": ([vp, vp], C.c_int),
        "psg_set_timing": ([vp, C.c_int], C.c_int),
        "psg_set_physics": ([vp, C.POINTER(CUnits), C.POINTER(RateTable), C.POINTER(XsTable), vp,
                             C.c_int, C.POINTER(Flags)], C.c_int),
        "psg_load_particles": ([vp, C.POINTER(Particles)], C.c_int),
        "psg_build_tree": ([vp, C.c_int], C.c_int),
        "psg_get_tree_info": ([vp, C.POINTER(TreeInfo)], C.c_int),
        "psg_get_tree": ([vp, vp, vp, vp, vp, vp], C.c_int),
        "psg_rt_trace": ([vp, vp, vp, C.c_float, C.POINTER(vp), C.POINTER(sz)], sz),
        "psg_trace": ([vp, vp, sz, vp, C.POINTER(vp), C.POINTER(sz)], C.c_int),
        "psg_run_ticks": ([vp, vp, sz, sz, i64, dbl, C.POINTER(TickStats)], C.c_int),
        "psg_run_ticks_device": ([vp, vp, sz, sz, i64, dbl, C.POINTER(TickStats)], C.c_int),
        "psg_get_state": ([vp, vp, vp, vp, vp], C.c_int),
        "psg_set_state": ([vp, vp, vp, vp], C.c_int),
        "psg_step_evolve": ([vp, vp, sz], C.c_int),
        "psg_set_sources": ([vp, vp, C.c_int, vp, C.c_int, C.c_uint64], C.c_int),
        "psg_get_sources": ([vp, vp, vp], C.c_int),
        "psg_emit_rays": ([vp, sz, sz, i64, dbl, vp], C.c_int),
        "psg_run_ticks_emit": ([vp, sz, sz, i64, dbl, C.POINTER(TickStats)], C.c_int),
        "psg_mlp_forward": ([vp, vp, vp, sz, vp], C.c_int),
        "psg_mlp_grad": ([vp, vp, vp, vp, sz, vp, vp], C.c_int),
        "psg_mlp_adam": ([vp, vp, vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int], C.c_int),
        "psg_set_update_log": ([vp, vp, sz, vp], C.c_int),
        "psg_set_surrogate": ([vp, vp, vp, vp, vp, vp, C.c_float], C.c_int),
        "psg_surrogate_forward": ([vp, vp, sz, vp], C.c_int),
        "psg_snapshot_write": ([C.c_char_p, C.POINTER(CSnapshot)], C.c_int),
        "psg_snapshot_read_header": ([C.c_char_p, C.POINTER(CSnapshot)], C.c_int),
        "psg_snapshot_read": ([C.c_char_p, C.POINTER(CSnapshot)], C.c_int),
        "psg_write_output": ([vp, C.c_char_p, C.POINTER(CSnapshot)], C.c_int),
        "psg_set_hits": ([vp, vp], C.c_int),
        "psg_set_recombination": ([vp, C.c_int, dbl, C.c_int, C.c_uint64], C.c_int),
        "psg_get_he_state": ([vp, vp, vp, vp, vp, vp], C.c_int),
        "psg_set_he_state": ([vp, vp, vp, vp, vp], C.c_int),
        "psg_secion_table_build": ([C.POINTER(CUnits), vp], C.c_int),
        "psg_get_rec_rays": ([vp, vp, vp, vp, sz, C.POINTER(sz)], C.c_int),
        "psg_get_rec_state": ([vp, vp, vp], C.c_int),
        "psg_set_rec_state": ([vp, vp, vp], C.c_int),
        "psg_set_tune": ([vp, C.POINTER(Tune)], C.c_int),
        "psg_get_tune": ([vp, C.POINTER(Tune)], C.c_int),
        "psg_autotune": ([vp, vp, sz, sz, i64, dbl, C.c_int, C.POINTER(Tune), C.POINTER(dbl)], C.c_int),
        "psg_device_arch": ([vp, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data


class Physics:
    """Units and tables, built by the library's host code from the reference's
    file formats (units_init, ar_init, xs_init, kernel.akline)."""

    def __init__(self, units, rates_path: str = RATES_HUI, kernel_path: str = KERNEL_AKLINE,
                 isothermal=True, on_the_spot=True, h_only=True, adiabatic=False, euler=False,
                 secondary_ionization=False):
        L = lib()
        self.units = units
        p = UnitParams(units.h, units.hmf, units.length_cmh, units.mass_gramh, units.time_sh)
        self.cu = CUnits()
        self._check(L.psg_units_init(C.byref(p), C.byref(self.cu)), "psg_units_init")
        self.ar = RateTable()
        self._check(L.psg_rate_table_load(rates_path.encode(), C.byref(self.cu), C.byref(self.ar)),
                    f"psg_rate_table_load({rates_path})")
        self.xs = XsTable()
        self._check(L.psg_xs_table_build(C.byref(self.cu), C.byref(self.xs)), "psg_xs_table_build")
        self.kernel = np.zeros(65536)
        n = C.c_int(0)
        self._check(L.psg_kernel_table_load(kernel_path.encode(), self.kernel.ctypes.data, 65536, C.byref(n)),
                    f"psg_kernel_table_load({kernel_path})")
        self.kernel = self.kernel[: n.value].copy()
        self.flags = Flags(int(isothermal), int(on_the_spot), int(h_only), int(adiabatic), int(euler),
                           int(secondary_ionization))

    @staticmethod
    def _check(rc, what):
        if rc != PSG_OK:
            raise PsgError(rc, what)

    def __del__(self):
        try:
            L = lib()
            L.psg_rate_table_free(C.byref(self.ar))
            L.psg_xs_table_free(C.byref(self.xs))
        except Exception:
            pass

    def ar_get(self, col: str, logT: float) -> float:
        return lib().psg_ar_get(C.byref(self.ar), AR_COLS.index(col), logT)

    def xs_get(self, species: str, freq: float) -> float:
        return lib().psg_xs_get(C.byref(self.xs), XS_SPECIES.index(species), freq)

    def sph_depth(self, r_h: float) -> float:
        return lib().psg_sph_depth(self.kernel.ctypes.data, len(self.kernel), r_h)

    def unit(self, name: str) -> float:
        return getattr(self.cu, name)

    def tables_for_oracle(self):
        """Raw table arrays (numpy views of the library's host tables)."""
        nr = self.ar.nrows
        ar_logT = np.ctypeslib.as_array(self.ar.logT, shape=(nr,)).copy()
        ar_cols = [np.ctypeslib.as_array(self.ar.col[i], shape=(nr,)).copy() for i in range(len(AR_COLS))]
        nx = self.xs.nrows
        xs_eng = np.ctypeslib.as_array(self.xs.eng, shape=(nx,)).copy()
        xs_HI = np.ctypeslib.as_array(self.xs.sigma[0], shape=(nx,)).copy()
        return dict(ar_nrows=nr, ar_min=self.ar.min, ar_step_inv=self.ar.step_inv, ar_logT=ar_logT,
                    ar_cols=ar_cols, xs_nrows=nx, xs_min=self.xs.min, xs_step_inv=self.xs.step_inv,
                    xs_cut_HI=self.xs.cut[0], xs_eng=xs_eng, xs_HI=xs_HI, kernel=self.kernel.copy())


class Context:
    """One device context (psg_context): particles, tree and state on a GPU."""

    def __init__(self, device: int = 0):
        L = lib()
        h = C.c_void_p()
        rc = L.psg_create(C.byref(h), device)
        if rc != PSG_OK:
            raise PsgError(rc, f"psg_create(device={device}): no usable CUDA device")
        self.h = h
        self.n = 0
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            lib().psg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != PSG_OK:
            msg = lib().psg_last_error(self.h)
            raise PsgError(rc, f"{what}: {msg.decode() if msg else ''}")

    def set_stream(self, stream_ptr: int | None):
        """Issue all work on the given cudaStream_t (an integer handle, e.g.
        torch.cuda.current_stream().cuda_stream); None restores the context's
        own stream."""
        self._check(lib().psg_set_stream(self.h, C.c_void_p(stream_ptr) if stream_ptr else None),
                    "psg_set_stream")

    def set_physics(self, phys: Physics):
        self.phys = phys
        self._check(lib().psg_set_physics(self.h, C.byref(phys.cu), C.byref(phys.ar), C.byref(phys.xs),
                                          phys.kernel.ctypes.data, len(phys.kernel), C.byref(phys.flags)),
                    "psg_set_physics")

    def load(self, f: Field, flag: np.ndarray | None = None):
        self._keep = [np.ascontiguousarray(a) for a in (f.pos, f.mass, f.sml, f.rho, f.ie, f.xHI, f.ye)]
        fl = None if flag is None else np.ascontiguousarray(flag, np.int8)
        p = Particles(f.n, *[a.ctypes.data for a in self._keep], _ptr(fl), f.boxsize)
        self._check(lib().psg_load_particles(self.h, C.byref(p)), "psg_load_particles")
        self.n = f.n

    def build_tree(self, ppc: int = 8):
        self._check(lib().psg_build_tree(self.h, int(ppc)), "psg_build_tree")

    def tree_info(self) -> dict:
        ti = TreeInfo()
        self._check(lib().psg_get_tree_info(self.h, C.byref(ti)), "psg_get_tree_info")
        return dict(ncells=ti.ncells, nleaves=ti.nleaves, skipped=ti.skipped, depth=ti.depth)

    def tree(self) -> dict:
        info = self.tree_info()
        nc = info["ncells"]
        bot = np.zeros((nc, 3), np.float32); top = np.zeros((nc, 3), np.float32)
        skip = np.zeros(nc, np.int32); pstart = np.zeros(nc + 1, np.int32)
        order = np.zeros(self.n - info["skipped"], np.int32)
        self._check(lib().psg_get_tree(self.h, bot.ctypes.data, top.ctypes.data, skip.ctypes.data,
                                       pstart.ctypes.data, order.ctypes.data), "psg_get_tree")
        return dict(bot=bot, top=top, skip=skip, pstart=pstart, order=order, **info)

    def rt_trace(self, s, d, dist) -> np.ndarray:
        """rt_trace(): one ray's hits sorted by (d, ipar)."""
        s = np.ascontiguousarray(s, np.float32); d = np.ascontiguousarray(d, np.float32)
        x = C.c_void_p(); size = C.c_size_t(0)
        n = lib().psg_rt_trace(self.h, s.ctypes.data, d.ctypes.data, C.c_float(dist), C.byref(x), C.byref(size))
        if n == C.c_size_t(-1).value:
            self._check(-2, "psg_rt_trace")
        out = np.zeros(n, XTYPE_DTYPE)
        if n:
            C.memmove(out.ctypes.data, x, n * XTYPE_DTYPE.itemsize)
        if x:
            C.CDLL(None).free(x)
        return out

    def trace(self, rays: np.ndarray):
        """trace(): all rays; returns (offsets[nray+1], hits)."""
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        off = np.zeros(len(rays) + 1, np.int64)
        x = C.c_void_p(); size = C.c_size_t(0)
        rc = lib().psg_trace(self.h, rays.ctypes.data, len(rays), off.ctypes.data, C.byref(x), C.byref(size))
        self._check(rc, "psg_trace")
        n = int(off[-1])
        out = np.zeros(n, XTYPE_DTYPE)
        if n:
            C.memmove(out.ctypes.data, x, n * XTYPE_DTYPE.itemsize)
        if x:
            C.CDLL(None).free(x)
        return off, out

    def run_ticks(self, rays: np.ndarray, nray_per_tick: int, nticks: int, first_tick: int,
                  tick_time: float) -> dict:
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        assert len(rays) == nray_per_tick * nticks
        st = TickStats()
        self._check(lib().psg_run_ticks(self.h, rays.ctypes.data, nray_per_tick, nticks, first_tick,
                                        tick_time, C.byref(st)), "psg_run_ticks")
        return _stats(st)

    def run_ticks_device(self, d_rays_ptr: int, nray_per_tick: int, nticks: int, first_tick: int,
                         tick_time: float) -> dict:
        st = TickStats()
        self._check(lib().psg_run_ticks_device(self.h, C.c_void_p(d_rays_ptr), nray_per_tick, nticks,
                                               first_tick, tick_time, C.byref(st)), "psg_run_ticks_device")
        return _stats(st)

    def set_sources(self, sources, spectra, seed: int):
        """sources: objects with pos, ngamma_dot (or a history: ticks +
        ngamma_dots), lastemit and optionally type/specid/dir/a/b/radius;
        spectra: list of (energies, weights)."""
        keep = []
        cs = (CSource * len(sources))()
        for c, src in zip(cs, sources):
            ticks = np.ascontiguousarray(getattr(src, "ticks", None) if getattr(src, "ticks", None) is not None
                                         else [0], np.int64)
            ngd = np.ascontiguousarray(getattr(src, "ngamma_dots", None) if getattr(src, "ngamma_dots", None)
                                       is not None else [src.ngamma_dot], np.float64)
            keep += [ticks, ngd]
            c.type = int(getattr(src, "type", SRC_POINT))
            c.specid = int(getattr(src, "specid", 0))
            c.pos[:] = [float(v) for v in src.pos]
            for name in ("dir", "a", "b"):
                v = getattr(src, name, None)
                if v is not None:
                    getattr(c, name)[:] = [float(x) for x in v]
            c.radius = float(getattr(src, "radius", 0.0))
            c.ticks, c.ngamma_dot, c.nhist = ticks.ctypes.data, ngd.ctypes.data, len(ticks)
            c.lastemit = int(src.lastemit)
        sp = (CSpectrum * len(spectra))()
        for c, (eng, wt) in zip(sp, spectra):
            e = np.ascontiguousarray(eng, np.float64); w = np.ascontiguousarray(wt, np.float64)
            keep += [e, w]
            c.eng, c.weight, c.n = e.ctypes.data, w.ctypes.data, len(e)
        self._check(lib().psg_set_sources(self.h, C.cast(cs, C.c_void_p), len(sources), C.cast(sp, C.c_void_p),
                                          len(spectra), C.c_uint64(seed)), "psg_set_sources")
        self.nsrc = len(sources)

    def sources_state(self):
        lastemit = np.zeros(self.nsrc, np.int64); cursor = np.zeros(self.nsrc, np.int32)
        self._check(lib().psg_get_sources(self.h, lastemit.ctypes.data, cursor.ctypes.data), "psg_get_sources")
        return lastemit, cursor

    def emit_rays(self, nray_per_tick: int, nticks: int, first_tick: int, tick_time: float) -> np.ndarray:
        out = np.zeros(nray_per_tick * nticks, RAY_DTYPE)
        self._check(lib().psg_emit_rays(self.h, nray_per_tick, nticks, first_tick, tick_time, out.ctypes.data),
                    "psg_emit_rays")
        return out

    def run_ticks_emit(self, nray_per_tick: int, nticks: int, first_tick: int, tick_time: float) -> dict:
        st = TickStats()
        self._check(lib().psg_run_ticks_emit(self.h, nray_per_tick, nticks, first_tick, tick_time, C.byref(st)),
                    "psg_run_ticks_emit")
        return _stats(st)

    def set_timing(self, on: bool):
        self._check(lib().psg_set_timing(self.h, int(bool(on))), "psg_set_timing")

    def state(self) -> dict:
        n = self.n
        lam = np.zeros(n); ie = np.zeros(n, np.float32); hits = np.zeros(n, np.int32); lh = np.zeros(n, np.int64)
        self._check(lib().psg_get_state(self.h, lam.ctypes.data, ie.ctypes.data, hits.ctypes.data,
                                        lh.ctypes.data), "psg_get_state")
        return dict(lambdaH=lam, ie=ie, hits=hits, lasthit=lh)

    def lambdaH(self, out: np.ndarray | None = None) -> np.ndarray:
        """x_HI of every particle (the result a tick produces), into `out`
        (float64[n], e.g. a view of pinned host memory) if given."""
        lam = np.zeros(self.n) if out is None else out
        assert lam.dtype == np.float64 and lam.shape == (self.n,) and lam.flags["C_CONTIGUOUS"]
        self._check(lib().psg_get_state(self.h, lam.ctypes.data, None, None, None), "psg_get_state")
        return lam

    def set_state(self, lambdaH=None, ie=None, lasthit=None):
        keep = [None if lambdaH is None else np.ascontiguousarray(lambdaH, np.float64),
                None if ie is None else np.ascontiguousarray(ie, np.float32),
                None if lasthit is None else np.ascontiguousarray(lasthit, np.int64)]
        self._check(lib().psg_set_state(self.h, *[_ptr(a) for a in keep]), "psg_set_state")

    def write_output(self, path: str, ids=None, src_pos=None, ngammas=None, **consts):
        """psystem_write_output(): the device state as a psphray-format file."""
        s = CSnapshot(ngas=self.n, nsrc=0 if src_pos is None else len(src_pos))
        for k in SNAP_CONSTS:
            setattr(s, k, float(consts.get(k, 0.0)))
        keep = []
        if ids is not None:
            keep.append(np.ascontiguousarray(ids, np.int64)); s.id = keep[-1].ctypes.data
        if src_pos is not None:
            keep += [np.ascontiguousarray(src_pos, np.float32), np.ascontiguousarray(ngammas, np.float64)]
            s.src_pos, s.ngammas = keep[-2].ctypes.data, keep[-1].ctypes.data
        self._check(lib().psg_write_output(self.h, path.encode(), C.byref(s)), "psg_write_output")

    def set_hits(self, hits):
        h = np.ascontiguousarray(hits, np.int32)
        self._check(lib().psg_set_hits(self.h, h.ctypes.data), "psg_set_hits")

    def set_recombination(self, nrec: int = 100, threshold: float = 0.1, disable_lte: bool = False, seed: int = 0):
        """Recombination rays when not on the spot (epoch nrec,
        psphray.recombineThreshold, psphray.disableLTE)."""
        self._check(lib().psg_set_recombination(self.h, int(nrec), float(threshold), int(bool(disable_lte)),
                                                C.c_uint64(seed)), "psg_set_recombination")

    def rec_rays(self, types: bool = False):
        """The last tick's recombination rays and their emitters (caller
        index); with types=True also each ray's type (0 HII, 1 HeII, 2 HeIII)."""
        n = C.c_size_t(0)
        self._check(lib().psg_get_rec_rays(self.h, None, None, None, 0, C.byref(n)), "psg_get_rec_rays")
        rays = np.zeros(n.value, RAY_DTYPE); ipar = np.zeros(n.value, np.int64); typ = np.zeros(n.value, np.int32)
        if n.value:
            self._check(lib().psg_get_rec_rays(self.h, rays.ctypes.data, ipar.ctypes.data, typ.ctypes.data, n.value,
                                               C.byref(n)), "psg_get_rec_rays")
        return (rays, ipar, typ) if types else (rays, ipar)

    def he_state(self) -> dict:
        """Helium fractions (lambdaHeI = x_HeI, lambdaHeII = x_HeII), yeMET and
        the helium recombination photons yGrecHeII, yGrecHeIII."""
        a, b = np.zeros(self.n), np.zeros(self.n)
        c, d, e = (np.zeros(self.n, np.float32) for _ in range(3))
        self._check(lib().psg_get_he_state(self.h, *[x.ctypes.data for x in (a, b, c, d, e)]), "psg_get_he_state")
        return dict(lambdaHeI=a, lambdaHeII=b, yeMET=c, yGrecHeII=d, yGrecHeIII=e)

    def set_he_state(self, lambdaHeI=None, lambdaHeII=None, yGrecHeII=None, yGrecHeIII=None):
        keep = [None if v is None else np.ascontiguousarray(v, np.float64) for v in (lambdaHeI, lambdaHeII)]
        keep += [None if v is None else np.ascontiguousarray(v, np.float32) for v in (yGrecHeII, yGrecHeIII)]
        self._check(lib().psg_set_he_state(self.h, *[_ptr(a) for a in keep]), "psg_set_he_state")

    def rec_state(self):
        """yGrecHII and the tick each particle was last hit by a source ray."""
        yg = np.zeros(self.n, np.float32); mark = np.zeros(self.n, np.int32)
        self._check(lib().psg_get_rec_state(self.h, yg.ctypes.data, mark.ctypes.data), "psg_get_rec_state")
        return yg, mark

    def set_rec_state(self, yGrecHII=None, srcmark=None):
        keep = [None if yGrecHII is None else np.ascontiguousarray(yGrecHII, np.float32),
                None if srcmark is None else np.ascontiguousarray(srcmark, np.int32)]
        self._check(lib().psg_set_rec_state(self.h, *[_ptr(a) for a in keep]), "psg_set_rec_state")

    def tune(self) -> dict:
        t = Tune()
        self._check(lib().psg_get_tune(self.h, C.byref(t)), "psg_get_tune")
        return t.as_dict()

    def set_tune(self, **kw):
        t = Tune()
        self._check(lib().psg_get_tune(self.h, C.byref(t)), "psg_get_tune")
        for k, v in kw.items():
            setattr(t, k, int(v))
        self._check(lib().psg_set_tune(self.h, C.byref(t)), "psg_set_tune")

    def autotune(self, d_rays_ptr: int, nray_per_tick: int, nticks: int, first_tick: int, tick_time: float,
                 reps: int = 2) -> tuple[dict, float]:
        """psg_autotune on device rays: the kept shapes and their batch time (ms)."""
        t = Tune()
        ms = C.c_double(0.0)
        self._check(lib().psg_autotune(self.h, C.c_void_p(d_rays_ptr), nray_per_tick, nticks, first_tick, tick_time,
                                       int(reps), C.byref(t), C.byref(ms)), "psg_autotune")
        return t.as_dict(), ms.value

    def step_evolve(self, steps: np.ndarray) -> np.ndarray:
        steps = np.ascontiguousarray(steps, STEP_DTYPE)
        self._check(lib().psg_step_evolve(self.h, steps.ctypes.data, len(steps)), "psg_step_evolve")
        return steps
