"""ctypes driver of the CPU oracle -- TEST INFRASTRUCTURE.

Loads oracle/_build/liboracle_f32.so (REAL = float, the reference's REAL
arithmetic) or liboracle_f64.so (the FP64 twin) and runs a synthetic case
through the restated Fortran solvers.  Only tests/, __graft_entry__.smoke()
and bench.py's CPU baseline legs use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
BUILD = HERE / "_build"

_libs = {}


def build(quiet=True):
    subprocess.run(["make", "-C", str(HERE)], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def load(dtype=np.float32, libm=False):
    """the float oracle, its FP64 twin, or (libm=True) the float build whose
    exp/pow are libm's expf/powf instead of the shared comcot_math.h ones"""
    key = np.dtype(dtype).name + ("_libm" if libm else "")
    if key in _libs:
        return _libs[key]
    if libm and np.dtype(dtype) != np.float32:
        raise ValueError("the libm build is a float build")
    name = {"float32": "liboracle_f32.so", "float64": "liboracle_f64.so",
            "float32_libm": "liboracle_f32_libm.so"}[key]
    path = BUILD / name
    if not path.exists():
        build()
    lib = C.CDLL(str(path))
    lib.ocl_step.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double]
    lib.ocl_arrival_start.argtypes = [C.c_void_p, C.c_double]
    lib.ocl_run.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_void_p, C.c_void_p,
                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ocl_run.restype = C.c_int
    lib.ocl_run_from.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ocl_run_from.restype = C.c_int
    lib.ocl_set_threads.argtypes = [C.c_int]
    for fn in ("ocl_mass", "ocl_moment", "ocl_open", "ocl_change", "ocl_update", "ocl_maxamp"):
        getattr(lib, fn).argtypes = [C.c_void_p]
    lib.ocl_jnq.argtypes = [C.c_void_p, C.c_void_p]
    lib.ocl_jnz.argtypes = [C.c_void_p, C.c_void_p]
    lib.ocl_newq.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    lib.ocl_all_grid.argtypes = [C.c_void_p, C.c_int]
    lib.ocl_gauge.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double]
    lib.ocl_gauge.restype = C.c_double
    lib.ocl_pq_depth.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ocl_para.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                             C.c_void_p, C.c_void_p] + [C.c_void_p] * 7
    lib.ocl_rel_time.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                 C.POINTER(C.c_double)]
    lib.ocl_rel_time.restype = C.c_int
    lib.ocl_corners.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_double,
                                C.c_double, C.c_double, C.c_void_p]
    lib.ocl_okada.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                              C.c_double, C.c_void_p]
    lib.ocl_okada_apply.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                    C.c_double, C.c_double, C.c_void_p, C.c_void_p]
    lib.ocl_sponge.argtypes = [C.c_void_p]
    lib.ocl_edge_sc.argtypes = [C.c_void_p, C.c_void_p]
    lib.ocl_newq_sc.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    lib.ocl_jnz_sc.argtypes = [C.c_void_p, C.c_void_p]
    lib.ocl_sponge_coef.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p]
    lib.ocl_expf.argtypes = [C.c_float]
    lib.ocl_expf.restype = C.c_float
    lib.ocl_powf.argtypes = [C.c_float, C.c_float]
    lib.ocl_powf.restype = C.c_float
    _libs[key] = lib
    return lib


class OFault(C.Structure):
    """ocl_fault (comcot_oracle.h)"""
    _fields_ = [(n, C.c_double) for n in ("hh", "l", "w", "d", "th", "dl", "rd", "x0", "y0", "xo", "yo")] + [
        ("sw", C.c_int)]


def okada_apply(faults, laycord, nx, ny, x=None, y=None, dx=0.0, dy=0.0, z=None, h=None, dtype=np.float32):
    """GET_FLOOR_DEFORM restated: returns (z + sum of deformations, h - sum)"""
    lib = load(dtype)
    arr = (OFault * max(1, len(faults)))()
    for k, f in enumerate(faults):
        for key, v in f.items():
            setattr(arr[k], key, v)
    zz = np.array(np.zeros((ny, nx)) if z is None else z, dtype=dtype, order="C", copy=True)
    hh = np.array(np.zeros((ny, nx)) if h is None else h, dtype=dtype, order="C", copy=True)
    xa = np.ascontiguousarray(np.zeros(nx) if x is None else x, dtype=np.float64)
    ya = np.ascontiguousarray(np.zeros(ny) if y is None else y, dtype=np.float64)
    lib.ocl_okada_apply(C.addressof(arr), len(faults), laycord, nx, ny, xa.ctypes.data, ya.ctypes.data, dx, dy,
                        zz.ctypes.data, hh.ctypes.data)
    return zz, hh


class OLayer(C.Structure):
    _fields_ = ([(n, C.c_int) for n in ("id", "parent", "level", "nx", "ny", "laycord", "laygov", "linchk",
                                        "modscm", "fric_switch", "rel_size", "rel_time")]
                + [("corners", C.c_int * 4)]
                + [(n, C.c_double) for n in ("dt", "rx", "ry", "grx", "gry", "fric_coef")]
                + [(n, C.c_void_p) for n in ("r1", "r11", "r6", "r3", "r5", "r0", "r22", "r2", "r4", "h", "hp", "hq",
                                             "z1", "z2", "m1", "m2", "n1", "n2", "dz2", "xflux", "yflux",
                                             "zmax", "arrival", "spx", "spy")]
                + [("sc_option", C.c_int), ("sc_fix_top", C.c_int), ("pos", C.c_void_p), ("cxy", C.c_void_p)])


class OracleRun:
    """Oracle state for every layer of a case."""

    def __init__(self, case, dtype=np.float32, coefs64=None, libm=False):
        self.case = case
        self.dtype = np.dtype(dtype)
        self.lib = load(self.dtype, libm=libm)
        n = len(case.layers)
        self.arr = (OLayer * n)()
        self.keep = []
        self.fields = []
        for k, L in enumerate(case.layers):
            self.fields.append(self._fill(self.arr[k], L, k == 0, coefs64[k] if coefs64 else None))
        # arrival at the start: step 0 where a wet cell is already above the threshold
        self.lib.ocl_arrival_start(C.addressof(self.arr[0]), float(case.arrival_thr))
        self.steps_done = 0  # outer steps run so far (a later run() continues the count)

    def _a(self, x, dt=None):
        a = np.ascontiguousarray(x, dtype=dt or self.dtype)
        self.keep.append(a)
        return a

    def _fill(self, o, L, is_root, c64):
        d = self.dtype
        o.id, o.parent, o.level, o.nx, o.ny = L.id, L.parent, L.level, L.nx, L.ny
        o.laycord, o.laygov, o.linchk, o.modscm, o.fric_switch = L.laycord, L.laygov, L.linchk, L.modscm, L.fric_switch
        o.rel_size, o.rel_time = L.rel_size, L.rel_time
        for q in range(4):
            o.corners[q] = int(L.corners[q])
        o.dt, o.rx, o.ry, o.grx, o.gry, o.fric_coef = L.dt, L.rx, L.ry, L.grx, L.gry, L.fric_coef
        f = {}
        ny, nx = L.ny, L.nx
        c = c64 if c64 is not None else L.coefs
        if c is not None:
            for nm in ("r1", "r11", "r6", "r3", "r5", "r2", "r4"):
                f[nm] = self._a(getattr(c, nm))
            for nm in ("r0", "r22"):
                v = getattr(c, nm, None)
                f[nm] = self._a(v if v is not None else np.zeros(ny))
        else:
            for nm in ("r1", "r11", "r6", "r3", "r5", "r0", "r22"):
                f[nm] = self._a(np.zeros(ny))
            f["r2"] = self._a(np.zeros((ny, nx)))
            f["r4"] = self._a(np.zeros((ny, nx)))
        f["h"] = self._a(L.H)
        f["hp"] = self._a(L.hp if L.hp is not None else np.zeros((ny, nx)))
        f["hq"] = self._a(L.hq if L.hq is not None else np.zeros((ny, nx)))
        f["z1"] = self._a(L.Z0.astype(np.float32).copy())
        for nm in ("z2", "m1", "m2", "n1", "n2", "dz2"):
            f[nm] = self._a(np.zeros((ny, nx)))
        f["xflux"] = self._a(np.zeros(2 * nx))
        f["yflux"] = self._a(np.zeros(2 * ny))
        f["zmax"] = self._a(L.Z0.astype(np.float32).copy()) if is_root else None
        f["arrival"] = self._a(np.full((ny, nx), -1), np.int32) if is_root else None
        sp = getattr(L, "sponge", None)
        f["spx"] = self._a(sp[0]) if (is_root and sp is not None) else None
        f["spy"] = self._a(sp[1]) if (is_root and sp is not None) else None
        sc = getattr(L, "sc", None)
        o.sc_option = 1 if sc is not None else 0
        o.sc_fix_top = int(sc.fix_top) if sc is not None else 0
        f["pos"] = self._a(sc.pos, np.int32) if sc is not None else None
        f["cxy"] = self._a(sc.cxy) if sc is not None else None
        for nm, a in f.items():
            setattr(o, nm, a.ctypes.data if a is not None else None)
        return f

    def run(self, nsteps, threads=1, arrival=True, maxamp=True):
        """Runs the next nsteps outer steps (numbered on from earlier runs, so
        arrival steps are the forecast's); returns their gauge series
        [nsteps, ng]."""
        self.lib.ocl_set_threads(int(threads))
        root = self.arr[0]
        saved_z, saved_a = root.zmax, root.arrival
        if not maxamp:
            root.zmax = None
        if not arrival:
            root.arrival = None
        g = self.case.gauges
        ng = len(g)
        gl = np.array([x[0] for x in g] or [0], np.int32)
        gi = np.array([x[1] for x in g] or [0], np.int32)
        gj = np.array([x[2] for x in g] or [0], np.int32)
        gx = np.array([x[3] for x in g] or [0], np.float64)
        gy = np.array([x[4] for x in g] or [0], np.float64)
        ts = np.zeros((max(nsteps, 1), max(ng, 1)), self.dtype)
        rc = self.lib.ocl_run_from(C.addressof(self.arr), len(self.case.layers), self.steps_done + 1, int(nsteps),
                                   float(self.case.arrival_thr), ng, gl.ctypes.data, gi.ctypes.data,
                                   gj.ctypes.data, gx.ctypes.data, gy.ctypes.data, ts.ctypes.data)
        root.zmax, root.arrival = saved_z, saved_a
        if rc != 0:
            raise RuntimeError("oracle run failed")
        self.steps_done += int(nsteps)
        return ts[:nsteps, :ng]

    def layer(self, k=0):
        """Fortran (:,:,2) view of layer k after the last completed step."""
        f = self.fields[k]
        # after CHANGE / UPDATE the levels are equal; level 1 is the latest
        return {"z": f["z1"], "m": f["m1"], "n": f["n1"], "zmax": f["zmax"], "arrival": f["arrival"],
                "dz": f["dz2"]}


def sponge_coef(laycord, x, y, h, dtype=np.float32):
    """SPONGE_COEF (boundaries.f90:250-345): coefficient fields [ny, nx]"""
    lib = load(dtype)
    ny, nx = h.shape
    xa = np.ascontiguousarray(x, dtype=dtype)
    ya = np.ascontiguousarray(y, dtype=dtype)
    ha = np.ascontiguousarray(h, dtype=dtype)
    cx = np.zeros((ny, nx), dtype)
    cy = np.zeros((ny, nx), dtype)
    lib.ocl_sponge_coef(nx, ny, laycord, xa.ctypes.data, ya.ctypes.data, ha.ctypes.data, cx.ctypes.data,
                        cy.ctypes.data)
    return cx, cy
