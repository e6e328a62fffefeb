"""Host-side mirror of the reference driver's use of the GPU ABI.

``ReferenceSession`` makes exactly the calls comcot.f90 makes
(GCOMCOT_INIT_GPU, GCOMCOT_INIT_LAYER per layer, then per step MASS_LAUNCH,
OPENBD_LAUNCH, ALL_GRID_LAUNCH, MOMT_LAUNCH, MAXAMP_LAUNCH, GCOMCOT_GET_Z per
gauge, CUDA_UPDATE_LAYER), with the same argument meaning, so tests read like
the reference's own DEBUG_CORE comparisons.  ``drive`` runs the same sequence
inside the library (one call) for timing.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .synth import Case, LayerSpec

F32 = np.float32


def _f(v):
    return C.byref(C.c_float(float(v)))


def _i(v):
    return C.byref(C.c_int(int(v)))


class ReferenceSession:
    def __init__(self, case: Case, fusion: bool = True, arrival: bool = False, init_layers: bool = True,
                 host_cache: dict | None = None):
        """host_cache: a dict shared by sessions over the same layers; the
        Fortran-order arrays of a layer (all but its surface) are built once
        and kept there, as a Fortran caller holds them for the whole run"""
        self.lib = _lib.load()
        self.case = case
        self.lib.gcomcot_init_gpu_()
        self.lib.gcomcot_set_fusion(1 if fusion else 0)
        self._keep = []
        # the host arrays a Fortran caller already holds (LO%R1 ... LO%Z), built once
        self._host = {}
        for L in case.layers:
            key = (id(L.H), L.id)
            if host_cache is not None and key in host_cache:
                a = dict(host_cache[key])
                a["Z"] = np.ascontiguousarray(L.Z0, dtype=F32)
            else:
                a = self._host_arrays(L)
                if host_cache is not None:
                    host_cache[key] = a
            self._host[L.id] = a
        # arrival tracking starts once the outer layer is on the device
        self._arrival = arrival
        if init_layers:
            self.init_layers()

    def init_layers(self):
        """GCOMCOT_INIT_LAYER for layer 1 then every sub-layer
        (comcot.f90:281-296), then arrival tracking if asked for"""
        for L in self.case.layers:
            self._init_layer(L)
        if self._arrival:
            self.lib.gcomcot_set_arrival_(_i(self.case.root.id), _f(self.case.arrival_thr))

    def stream(self) -> int:
        return int(self.lib.gcomcot_stream() or 0)

    @staticmethod
    def _host_arrays(L: LayerSpec) -> dict:
        """the NX x NY Fortran-order host arrays GCOMCOT_INIT_LAYER and the
        extension calls read, as comcot.f90 holds them"""
        ny, nx = L.ny, L.nx
        full = lambda v: np.ascontiguousarray(np.repeat(np.asarray(v)[:, None], nx, axis=1), dtype=F32)
        a = {}
        if L.laycord == 1 or L.laygov != 0:
            a["hp"] = np.ascontiguousarray(L.hp, dtype=F32)
            a["hq"] = np.ascontiguousarray(L.hq, dtype=F32)
        if L.sc is not None:
            a["pos"] = np.ascontiguousarray(np.moveaxis(L.sc.pos, -1, 0), dtype=np.int32)
            a["cxy"] = np.ascontiguousarray(np.moveaxis(L.sc.cxy, -1, 0), dtype=F32)
        if L.laycord == 0 and L.laygov == 1:
            c = L.coefs
            a["r0"], a["r21"], a["r22"] = full(c.r0), full(c.r1), full(c.r22)
        if L.coefs is not None:
            c = L.coefs
            a["R1"], a["R11"], a["R3"], a["R5"] = full(c.r1), full(c.r11), full(c.r3), full(c.r5)
            a["R2"] = np.ascontiguousarray(c.r2, dtype=F32)
            a["R4"] = np.ascontiguousarray(c.r4, dtype=F32)
            a["R6"] = np.ascontiguousarray(c.r6, dtype=F32)
        else:
            z = np.zeros((ny, nx), F32)
            a["R1"] = a["R11"] = a["R3"] = a["R5"] = a["R2"] = a["R4"] = z
            a["R6"] = np.zeros(ny, F32)
        a["H"] = np.ascontiguousarray(L.H, dtype=F32)
        a["Z"] = np.ascontiguousarray(L.Z0, dtype=F32)
        a["corners"] = np.array(L.corners, dtype=np.int32)
        if L.sponge is not None:
            a["spx"] = np.ascontiguousarray(L.sponge[0], dtype=F32)
            a["spy"] = np.ascontiguousarray(L.sponge[1], dtype=F32)
        return a

    def _init_layer(self, L: LayerSpec):
        lib = self.lib
        ny, nx = L.ny, L.nx
        a = self._host[L.id]
        if L.laycord == 1 or L.laygov != 0:
            lib.gcomcot_set_layer_params_(_i(L.id), _i(L.laycord), _i(L.laygov), _f(L.dt), _f(L.rx), _f(L.ry),
                                          _f(L.grx), _f(L.gry), _i(L.fric_switch), _f(L.fric_coef),
                                          _i(L.linchk), _i(L.modscm), _i(nx), _i(ny), _lib.fptr(a["hp"]),
                                          _lib.fptr(a["hq"]))
        if L.sc is not None:
            # SC_OPTION = 1 tables in Fortran order POS(NX,NY,2), CXY(NX,NY,4)
            parent = next(Q for Q in self.case.layers if Q.id == L.parent)
            lib.gcomcot_set_sc_tables_(_i(L.id), _lib.iptr(a["pos"]), _lib.fptr(a["cxy"]), _i(nx), _i(ny),
                                       _i(parent.modscm), _i(1 if L.sc.fix_top else 0))
        if L.laycord == 0 and L.laygov == 1:
            lib.gcomcot_set_layer_coefs_(_i(L.id), _lib.fptr(a["r0"]), _lib.fptr(a["r21"]), _lib.fptr(a["r22"]),
                                         _i(nx), _i(ny))
        lib.gcomcot_init_layer_(_i(L.id), _i(L.parent), _i(L.level), _i(L.rel_size), _i(L.rel_time),
                                _lib.iptr(a["corners"]), _f(L.grx), _f(L.gry), _lib.fptr(a["R1"]),
                                _lib.fptr(a["R2"]), _lib.fptr(a["R3"]), _lib.fptr(a["R4"]), _lib.fptr(a["R5"]),
                                _lib.fptr(a["R6"]), _lib.fptr(a["R11"]), _lib.fptr(a["H"]), _lib.fptr(a["Z"]),
                                _i(nx), _i(ny))
        if L.sponge is not None:
            # BC_TYPE 1: SPONGE_COEF's fields (comcot.f90:220)
            lib.gcomcot_set_sponge_(_i(L.id), _lib.fptr(a["spx"]), _lib.fptr(a["spy"]), _f(L.dt), _i(nx), _i(ny))

    # ---- one outer step exactly as comcot.f90:359-439 ----
    def step(self, maxamp: bool = True):
        lib, rid = self.lib, self.case.root.id
        lib.mass_launch_(None, None, None, _i(rid))
        lib.openbd_launch_(None)
        if len(self.case.layers) > 1:
            lib.all_grid_launch_()
        lib.momt_launch_(None, None, None, _i(rid))
        if self.case.root.sponge is not None:
            lib.sponge_launch_(_i(rid))
        if maxamp:
            lib.maxamp_launch_(_i(rid))
        ts = [self.get_ts(g) for g in self.case.gauges]
        lib.cuda_update_layer_(_i(rid))
        return ts

    def get_ts(self, gauge):
        """GET_TS: bilinear interpolation of the 2x2 stencil (output.f90:1078-1090)."""
        lid, ki, kj, cx, cy = gauge
        l = [C.c_float() for _ in range(4)]
        self.lib.gcomcot_get_z_(_i(lid), *[C.byref(v) for v in l], _i(ki), _i(kj))
        l1, l2, l3, l4 = (F32(v.value) for v in l)
        cx, cy = F32(cx), F32(cy)
        one = F32(1.0)
        return float(l1 * (one - cx) * (one - cy) + l2 * cx * (one - cy) + l3 * (one - cx) * cy + l4 * cx * cy)

    def drive(self, nsteps: int, maxamp: bool = True):
        """The same sequence issued from inside the library; returns the raw
        2x2 gauge stencils [nsteps, ngauges, 4]."""
        g = self.case.gauges
        ng = len(g)
        gl = np.array([x[0] for x in g] or [0], dtype=np.int32)
        gi = np.array([x[1] for x in g] or [0], dtype=np.int32)
        gj = np.array([x[2] for x in g] or [0], dtype=np.int32)
        out = np.zeros((max(nsteps, 1), max(ng, 1), 4), dtype=F32)
        rc = self.lib.gcomcot_drive(nsteps, 1 if maxamp else 0, ng, _lib.iptr(gl), _lib.iptr(gi), _lib.iptr(gj),
                                    _lib.fptr(out))
        if rc != 0:
            raise RuntimeError(f"gcomcot_drive failed: {rc}")
        return out[:nsteps, :ng]

    # ---- whole-field reads (Fortran Z(:,:,2), M(:,:,2), N(:,:,2)) ----
    def _layer(self, lid):
        return next(L for L in self.case.layers if L.id == lid)

    def getz(self, lid=1):
        L = self._layer(lid)
        z = np.zeros((L.ny, L.nx), F32)
        self.lib.cuda_getz_(_lib.fptr(z), _i(lid))
        return z

    def getmn(self, lid=1):
        L = self._layer(lid)
        m = np.zeros((L.ny, L.nx), F32)
        n = np.zeros((L.ny, L.nx), F32)
        self.lib.cuda_getmn_(_lib.fptr(m), _lib.fptr(n), _i(lid))
        return m, n

    def getzmax(self, lid=1):
        L = self._layer(lid)
        z = np.zeros((L.ny, L.nx), F32)
        self.lib.cuda_getzmax_(_lib.fptr(z), _i(lid))
        return z

    def getarrival(self, lid=1):
        L = self._layer(lid)
        a = np.zeros((L.ny, L.nx), np.int32)
        self.lib.gcomcot_get_arrival_(_lib.iptr(a), _i(lid))
        return a

    def launches(self):
        return int(self.lib.gcomcot_launch_count())

    def close(self):
        self.lib.cuda_shutdown_()
