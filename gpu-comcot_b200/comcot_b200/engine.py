"""Python front of the batched ensemble / serving engine (gc_engine_* in
include/gcomcot.h).  A member is a linear-spherical forecast, optionally with
one nested child layer; members built on the same bathymetry (and the same
child) share one grid class."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .synth import Case

F32 = np.float32


class PinnedPool:
    """page-locked host blocks (gc_host_alloc) reused by size, so results
    can be copied from the device while the host goes on"""

    def __init__(self, lib):
        self.lib = lib
        self.free = {}

    def take(self, nbytes: int) -> int:
        blocks = self.free.get(nbytes)
        if blocks:
            return blocks.pop()
        ptr = self.lib.gc_host_alloc(int(nbytes))
        if not ptr:
            raise MemoryError("page-locked host memory refused")
        return ptr

    def give(self, nbytes: int, ptr: int):
        self.free.setdefault(nbytes, []).append(ptr)

    def close(self):
        for blocks in self.free.values():
            for ptr in blocks:
                self.lib.gc_host_free(ptr)
        self.free.clear()


class PendingRead:
    """results on their way from the device (Engine.read_async)"""

    def __init__(self, lib, pool, event, ptr, nbytes, views):
        self.lib, self.pool, self.event, self.ptr, self.nbytes, self.views = lib, pool, event, ptr, nbytes, views

    def done(self) -> bool:
        rc = self.lib.gc_event_query(self.event)
        if rc < 0:
            raise RuntimeError(f"gc_event_query failed: {rc}")
        return rc == 1

    def take(self) -> dict:
        """waits for the copies, returns the results as ordinary arrays and
        gives the page-locked block back to the pool"""
        rc = self.lib.gc_event_wait(self.event)
        if rc != 0:
            raise RuntimeError(f"gc_event_wait failed: {rc}")
        out = {k: np.array(v, copy=True) for k, v in self.views.items()}
        self.lib.gc_event_release(self.event)
        self.pool.give(self.nbytes, self.ptr)
        self.event = None
        return out


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
        self._axes = set()
        self.pinned = PinnedPool(self.lib)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def close(self):
        if self.h:
            self.lib.gc_engine_destroy(self.h)
            self.h = None
            self.pinned.close()

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

    def add_faults(self, case: Case, faults, nsteps=None, gauges=None, arrival_thr=None) -> int:
        """a member whose initial state is generated on the device from fault
        parameters (list of dicts with gc_fault's keys) on case.root's grid"""
        L = case.root
        cls = self.add_class(L)
        if cls not in self._axes:
            x = np.ascontiguousarray(L.x, dtype=F32)
            y = np.ascontiguousarray(L.y, dtype=F32)
            rc = self.lib.gc_engine_set_class_axes(self.h, cls, _lib.fptr(x), _lib.fptr(y))
            if rc != 0:
                raise RuntimeError(f"gc_engine_set_class_axes failed: {rc}")
            self._axes.add(cls)
        g = case.gauges if gauges is None else gauges
        ng = len(g)
        gij = np.array([[x[1], x[2]] for x in g] or [[0, 0]], dtype=np.int32)
        gw = np.array([[x[3], x[4]] for x in g] or [[0, 0]], dtype=F32)
        n = case.nsteps if nsteps is None else nsteps
        thr = case.arrival_thr if arrival_thr is None else arrival_thr
        arr = _lib.faults_array(faults)
        rc = self.lib.gc_engine_add_member_faults(self.h, cls, C.cast(arr, C.c_void_p), len(faults), int(n), ng,
                                                  _lib.iptr(gij), _lib.fptr(gw), C.c_float(thr))
        if rc == -2:
            raise MemoryError("engine budget exhausted")
        if rc < 0:
            raise RuntimeError(f"gc_engine_add_member_faults failed: {rc}")
        self.members[rc] = (L.nx, L.ny, n, ng, None)
        return rc

    def add_nested_class(self, P, Cl) -> int:
        """class for outer layer P with child layer Cl (a LayerSpec with parent P)"""
        key = (id(P.H), id(Cl.H), tuple(Cl.corners), Cl.rel_size, Cl.rel_time)
        if key in self.classes:
            return self.classes[key][0]
        pcls = self.add_class(P)
        d = _lib.ChildDesc()
        d.nx, d.ny = Cl.nx, Cl.ny
        for q in range(4):
            d.corners[q] = int(Cl.corners[q])
        d.rel_size, d.rel_time = Cl.rel_size, Cl.rel_time
        d.laycord, d.laygov, d.linchk, d.modscm, d.fric_switch = (Cl.laycord, Cl.laygov, Cl.linchk, Cl.modscm,
                                                                  Cl.fric_switch)
        d.dt, d.rx, d.ry, d.grx, d.gry, d.fric_coef = Cl.dt, Cl.rx, Cl.ry, Cl.grx, Cl.gry, Cl.fric_coef
        keep = [np.ascontiguousarray(Cl.H, dtype=F32)]
        d.h = _lib.fptr(keep[0])
        if Cl.hp is not None and Cl.hq is not None:
            keep += [np.ascontiguousarray(Cl.hp, dtype=F32), np.ascontiguousarray(Cl.hq, dtype=F32)]
            d.hp, d.hq = _lib.fptr(keep[1]), _lib.fptr(keep[2])
        if Cl.coefs is not None:
            keep.append(np.ascontiguousarray(Cl.coefs.rows(), dtype=F32))
            d.rows = _lib.fptr(keep[-1])
            if Cl.laycord == 0 and Cl.laygov == 1:
                keep.append(np.ascontiguousarray(np.stack([Cl.coefs.r0, Cl.coefs.r22]), dtype=F32))
                d.rows2 = _lib.fptr(keep[-1])
        if Cl.sc is not None:
            # SC_OPTION = 1 tables, [ny][nx][2] and [ny][nx][4]
            keep += [np.ascontiguousarray(Cl.sc.pos, dtype=np.int32), np.ascontiguousarray(Cl.sc.cxy, dtype=F32)]
            d.sc_pos, d.sc_cxy = _lib.iptr(keep[-2]), _lib.fptr(keep[-1])
            d.sc_fix_top = 1 if Cl.sc.fix_top else 0
        d.parent_modscm = P.modscm
        rc = self.lib.gc_engine_add_nested_class(self.h, pcls, C.byref(d))
        if rc == -2:
            raise MemoryError("engine budget exhausted")
        if rc < 0:
            raise RuntimeError(f"gc_engine_add_nested_class failed: {rc}")
        self.classes[key] = (rc, P.nx, P.ny)
        return rc

    def add(self, case: Case, z0=None, cls=None, nsteps=None, gauges=None, arrival_thr=None, child_z0=None) -> int:
        """adds the case as a member; a two-layer case becomes a nested member.
        Gauges are (layer_id, KI, KJ, CX, CY) with KI, KJ 1-based in that layer."""
        L = case.root
        nested = len(case.layers) > 1
        if len(case.layers) > 2:
            raise ValueError("the engine runs at most one child layer per member")
        if cls is None:
            cls = self.add_nested_class(L, case.layers[1]) if nested else self.add_class(L)
        z0 = np.ascontiguousarray(L.Z0 if z0 is None else z0, dtype=F32)
        g = case.gauges if gauges is None else gauges
        ng = len(g)
        gij = np.array([[x[1], x[2]] for x in g] or [[0, 0]], dtype=np.int32)
        gw = np.array([[x[3], x[4]] for x in g] or [[0, 0]], dtype=F32)
        n = case.nsteps if nsteps is None else nsteps
        thr = case.arrival_thr if arrival_thr is None else arrival_thr
        if nested:
            Cl = case.layers[1]
            gl = np.array([0 if x[0] == L.id else 1 for x in g] or [0], dtype=np.int32)
            cz = np.ascontiguousarray(Cl.Z0 if child_z0 is None else child_z0, dtype=F32)
            rc = self.lib.gc_engine_add_nested_member(self.h, cls, _lib.fptr(z0), _lib.fptr(cz), int(n), ng,
                                                      _lib.iptr(gl), _lib.iptr(gij), _lib.fptr(gw), C.c_float(thr))
        else:
            if any(x[0] != L.id for x in g):
                raise ValueError("gauge on a layer the case does not have")
            rc = self.lib.gc_engine_add_member(self.h, cls, _lib.fptr(z0), int(n), ng, _lib.iptr(gij),
                                               _lib.fptr(gw), C.c_float(thr))
        if rc == -2:
            raise MemoryError("engine budget exhausted")
        if rc < 0:
            raise RuntimeError(f"gc_engine_add_member failed: {rc}")
        child = (case.layers[1].nx, case.layers[1].ny) if nested else None
        self.members[rc] = (L.nx, L.ny, n, ng, child)
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

    def idle(self) -> bool:
        """True when everything issued so far has finished (does not wait)"""
        rc = self.lib.gc_engine_query(self.h)
        if rc < 0:
            raise RuntimeError(f"gc_engine_query failed: {rc}")
        return rc == 1

    def done(self, mid: int) -> bool:
        return self.lib.gc_engine_member_done(self.h, mid) == 1

    def steps_done(self, mid: int) -> int:
        """outer steps the member has been issued (complete after sync())"""
        rc = self.lib.gc_engine_member_steps(self.h, mid)
        if rc < 0:
            raise RuntimeError(f"gc_engine_member_steps failed: {rc}")
        return rc

    def read(self, mid: int, fields=("z", "m", "n", "zmax", "arrival", "ts")) -> dict:
        """results of a member (the named fields only); nested members also
        give child_z/child_m/child_n when "child" is among the fields or the
        default set is asked for"""
        nx, ny, n, ng, child = self.members[mid]
        want = set(fields)
        out = {}
        for k in ("z", "m", "n", "zmax"):
            if k in want:
                out[k] = np.zeros((ny, nx), F32)
        if "arrival" in want:
            out["arrival"] = np.zeros((ny, nx), np.int32)
        if "ts" in want:
            out["ts"] = np.zeros((n, max(ng, 1)), F32)
        rc = self.lib.gc_engine_read(self.h, mid, _lib.fptr(out.get("z")), _lib.fptr(out.get("m")),
                                     _lib.fptr(out.get("n")), _lib.fptr(out.get("zmax")),
                                     _lib.iptr(out.get("arrival")), _lib.fptr(out["ts"]) if ng and "ts" in want
                                     else None)
        if rc != 0:
            raise RuntimeError(f"gc_engine_read failed: {rc}")
        if "ts" in out:
            out["ts"] = out["ts"][:, :ng]
        if child is not None and ("child" in want or "z" in want):
            cnx, cny = child
            for k in ("child_z", "child_m", "child_n"):
                out[k] = np.zeros((cny, cnx), F32)
            rc = self.lib.gc_engine_read_child(self.h, mid, _lib.fptr(out["child_z"]), _lib.fptr(out["child_m"]),
                                               _lib.fptr(out["child_n"]))
            if rc != 0:
                raise RuntimeError(f"gc_engine_read_child failed: {rc}")
        return out

    def read_async(self, mid: int, fields=("zmax", "arrival", "ts")) -> PendingRead:
        """the named results (z, m, n, zmax, arrival, ts) copied into
        page-locked host memory behind the member's issued steps; the host
        goes on at once.  The member may be released right after."""
        nx, ny, n, ng, _child = self.members[mid]
        shapes = {"z": ((ny, nx), F32), "m": ((ny, nx), F32), "n": ((ny, nx), F32), "zmax": ((ny, nx), F32),
                  "arrival": ((ny, nx), np.int32), "ts": ((n, ng), F32)}
        want = [k for k in ("z", "m", "n", "zmax", "arrival", "ts") if k in fields and not (k == "ts" and ng == 0)]
        offs, total = {}, 0
        for k in want:
            shape, dt = shapes[k]
            offs[k] = total
            total += (int(np.prod(shape)) * np.dtype(dt).itemsize + 255) // 256 * 256
        total = max(total, 256)
        ptr = self.pinned.take(total)
        views = {}
        for k in want:
            shape, dt = shapes[k]
            cnt = int(np.prod(shape))
            buf = (C.c_byte * (cnt * np.dtype(dt).itemsize)).from_address(ptr + offs[k])
            views[k] = np.frombuffer(buf, dtype=dt, count=cnt).reshape(shape)
        ptrs = {k: (views[k].ctypes.data_as(_lib.P_I if k == "arrival" else _lib.P_F) if k in views else None)
                for k in shapes}
        ev = C.c_void_p()
        rc = self.lib.gc_engine_read_async(self.h, mid, ptrs["z"], ptrs["m"], ptrs["n"], ptrs["zmax"],
                                           ptrs["arrival"], ptrs["ts"], C.byref(ev))
        if rc != 0:
            self.pinned.give(total, ptr)
            raise RuntimeError(f"gc_engine_read_async failed: {rc}")
        return PendingRead(self.lib, self.pinned, ev, ptr, total, views)

    def release(self, mid: int):
        rc = self.lib.gc_engine_release(self.h, mid)
        if rc != 0:
            raise RuntimeError(f"gc_engine_release failed: {rc}")
        self.members.pop(mid, None)

    def health(self, mid: int, bound: float = 100.0) -> int:
        """0 healthy; bit 0: a NaN/Inf appeared; bit 1: |eta| > bound metres"""
        rc = self.lib.gc_engine_member_health(self.h, mid, C.c_float(bound))
        if rc < 0:
            raise RuntimeError(f"gc_engine_member_health failed: {rc}")
        return rc

    def autotune(self, reps=5) -> int:
        return self.lib.gc_engine_autotune(self.h, int(reps))

    def prepare(self):
        """builds the work list and the step-chunk graph now, so that the
        next step() does not pay for them"""
        rc = self.lib.gc_engine_prepare(self.h)
        if rc < 0:
            raise RuntimeError(f"gc_engine_prepare failed: {rc}")

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
