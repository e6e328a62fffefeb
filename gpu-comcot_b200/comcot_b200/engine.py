"""Python front of the batched ensemble / serving engine (gc_engine_* in
include/gcomcot.h).  Members are linear-spherical single-layer forecasts;
members built on the same bathymetry share one grid class."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .synth import Case

F32 = np.float32


class Engine:
    def __init__(self, budget: int):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.gc_engine_create(int(budget), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"gc_engine_create failed: {rc}")
        self.h = h
        self.classes = {}
        self.members = {}

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def close(self):
        if self.h:
            self.lib.gc_engine_destroy(self.h)
            self.h = None

    def config(self, variant=-1, use_graphs=1, chunk=32):
        rc = self.lib.gc_engine_config(self.h, int(variant), int(use_graphs), int(chunk))
        if rc != 0:
            raise RuntimeError(f"gc_engine_config failed: {rc}")

    def add_class(self, L) -> int:
        key = id(L.H)
        if key in self.classes:
            return self.classes[key][0]
        H = np.ascontiguousarray(L.H, dtype=F32)
        rows = np.ascontiguousarray(L.coefs.rows(), dtype=F32)
        rc = self.lib.gc_engine_add_class(self.h, L.nx, L.ny, _lib.fptr(H), _lib.fptr(rows))
        if rc == -2:
            raise MemoryError("engine budget exhausted")
        if rc < 0:
            raise RuntimeError(f"gc_engine_add_class failed: {rc}")
        self.classes[key] = (rc, L.nx, L.ny)
        return rc

    def add(self, case: Case, z0=None, cls=None, nsteps=None, gauges=None, arrival_thr=None) -> int:
        L = case.root
        if cls is None:
            cls = self.add_class(L)
        z0 = np.ascontiguousarray(L.Z0 if z0 is None else z0, dtype=F32)
        g = case.gauges if gauges is None else gauges
        ng = len(g)
        gij = np.array([[x[1], x[2]] for x in g] or [[0, 0]], dtype=np.int32)
        gw = np.array([[x[3], x[4]] for x in g] or [[0, 0]], dtype=F32)
        n = case.nsteps if nsteps is None else nsteps
        thr = case.arrival_thr if arrival_thr is None else arrival_thr
        rc = self.lib.gc_engine_add_member(self.h, cls, _lib.fptr(z0), int(n), ng, _lib.iptr(gij), _lib.fptr(gw),
                                           C.c_float(thr))
        if rc == -2:
            raise MemoryError("engine budget exhausted")
        if rc < 0:
            raise RuntimeError(f"gc_engine_add_member failed: {rc}")
        self.members[rc] = (L.nx, L.ny, n, ng)
        return rc

    def step(self, n: int) -> int:
        rc = self.lib.gc_engine_step(self.h, int(n))
        if rc < 0:
            raise RuntimeError(f"gc_engine_step failed: {rc}")
        return rc

    def sync(self):
        rc = self.lib.gc_engine_sync(self.h)
        if rc != 0:
            raise RuntimeError(f"gc_engine_sync failed: {rc}")

    def done(self, mid: int) -> bool:
        return self.lib.gc_engine_member_done(self.h, mid) == 1

    def read(self, mid: int) -> dict:
        nx, ny, n, ng = self.members[mid]
        out = {k: np.zeros((ny, nx), F32) for k in ("z", "m", "n", "zmax")}
        out["arrival"] = np.zeros((ny, nx), np.int32)
        out["ts"] = np.zeros((n, max(ng, 1)), F32)
        rc = self.lib.gc_engine_read(self.h, mid, _lib.fptr(out["z"]), _lib.fptr(out["m"]), _lib.fptr(out["n"]),
                                     _lib.fptr(out["zmax"]), _lib.iptr(out["arrival"]),
                                     _lib.fptr(out["ts"]) if ng else None)
        if rc != 0:
            raise RuntimeError(f"gc_engine_read failed: {rc}")
        out["ts"] = out["ts"][:, :ng]
        return out

    def release(self, mid: int):
        rc = self.lib.gc_engine_release(self.h, mid)
        if rc != 0:
            raise RuntimeError(f"gc_engine_release failed: {rc}")
        self.members.pop(mid, None)

    def autotune(self, reps=5) -> int:
        return self.lib.gc_engine_autotune(self.h, int(reps))

    def variant(self) -> int:
        return self.lib.gc_engine_variant(self.h)

    def bytes_in_use(self) -> int:
        return int(self.lib.gc_engine_bytes_in_use(self.h))

    def member_bytes(self, cls: int) -> int:
        return int(self.lib.gc_engine_member_bytes(self.h, cls))

    def launches(self) -> int:
        return int(self.lib.gc_engine_launches(self.h))

    def stream(self) -> int:
        """cudaStream_t (as an int) the engine launches on"""
        return int(self.lib.gc_engine_stream(self.h) or 0)
