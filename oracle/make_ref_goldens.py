#!/usr/bin/env python
"""Golden vectors from the reference's own CUDA kernels -- TEST INFRASTRUCTURE.

The reference ships no fixtures and its Fortran cannot be compiled here, so the
CPU oracle is pinned against outputs of the reference's CUDA kernels, built from
their sources by oracle/ref.mk (two builds: the reference's default FMA
contraction, and -fmad=false) and driven through the reference's C ABI.  Run on a
GPU machine:

    make -C oracle -f ref.mk && python oracle/make_ref_goldens.py

Cases (one parent 186 x 144 linear spherical layer, one 129 x 129 child with
ratio 4 at corners (20,51,20,51)); every size below was chosen so that the
reference kernels neither read outside their arrays nor run a full-mask warp
shuffle with lanes diverged (checked by reading the kernels):
  mass    -- mass_kernel (GPUMass_s.cu:39-102); NX = 186 is a multiple of the
             62 rows a block covers, so no block reads past row NX
  maxamp  -- maximum_recorder_kernel (GPUOutput.cu:46-53) after that mass
  jnq     -- edgeinterp_vert2/hori2 at T = 1 (GPUall_grids.cu:184-297); the
             parent extends >= 120 cells past the child corners, which the edge
             kernels' unguarded loads need
  newq2/3 -- the same kernels at T = 2 (forecast cached) and T = 3 (cache blend)
  jnz     -- jnz_wrap_based_kernel<4> (GPUall_grids.cu:487-585); child
             NX - 1 = 128 is a multiple of the 64-thread blocks, so no thread
             returns early before the warp reductions
The momentum and open-boundary kernels are not run: they issue full-mask
shuffles inside lane-dependent guards (GPUMoment_s.cu:93-138,
GPUOpen_BD.cu:57-170), which is undefined behaviour on this architecture.

Output: tests/golden/ref_kernels.npz (inputs and both builds' outputs).
"""
from __future__ import annotations

import ctypes as C
import json
import os
import pathlib
import subprocess
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parent
OUT = pathlib.Path(os.environ.get("GOLDEN_OUT", str(ROOT / "tests" / "golden" / "ref_kernels.npz")))

PNX, PNY = 186, 144
CORNERS = [20, 51, 20, 51]
RS = 4
CNX = (CORNERS[1] - CORNERS[0] + 1) * RS + 1
CNY = (CORNERS[3] - CORNERS[2] + 1) * RS + 1
REL_TIME = 3   # odd: JNZ averages Z2 only (all_grids.f90:385-390)


def make_inputs():
    """deterministic parent/child states (numpy float32, [ny, nx])"""
    sys.path.insert(0, str(ROOT / "gpu-comcot_b200"))
    sys.path.insert(0, str(HERE))
    from comcot_b200 import precompute as pc
    from comcot_b200 import synth
    import oracle

    case = synth.single_layer_case("ref", PNX, PNY, 2.0, 2.0, 0, seed=77, n_seamounts=6, shelf_cols=20,
                                   land_cols=6, source="dipole", amp=3.0)
    P = case.root
    o = oracle.OracleRun(case)
    o.run(25, arrival=False)                      # a developed wave field
    st = o.fields[0]
    z1 = st["z1"].copy()
    m1 = st["m1"].copy()
    n1 = st["n1"].copy()
    # one more mass + open so Z2 differs from Z1 (NEWQ and JNZ read Z2)
    o.lib.ocl_mass(C.addressof(o.arr[0]))
    o.lib.ocl_open(C.addressof(o.arr[0]))
    z2 = st["z2"].copy()
    rng = np.random.default_rng(5)
    # child: shelf with land and shoals, and a surface with dry spots
    cx = np.linspace(0, 1, CNX)[None, :]
    cy = np.linspace(0, 1, CNY)[:, None]
    hc = (150.0 - 180.0 * cx + 20.0 * np.sin(7 * cx + 3 * cy)).astype(np.float32)
    zc1 = (0.3 * np.sin(5 * cx) * np.cos(4 * cy)).astype(np.float32)
    zc2 = (zc1 + 0.05 * np.cos(6 * cx + cy)).astype(np.float32)
    zc1 = np.where(hc + zc1 <= 1e-5, -hc, zc1).astype(np.float32)
    zc2 = np.where(hc + zc2 <= 1e-5, -hc, zc2).astype(np.float32)
    c = P.coefs
    return {
        "p_h": P.H, "p_z1": z1, "p_z2": z2, "p_m1": m1, "p_n1": n1, "p_zmax": P.Z0.astype(np.float32),
        "p_r1": c.r1, "p_r11": c.r11, "p_r6": c.r6, "p_r3": c.r3, "p_r5": c.r5, "p_r2": c.r2, "p_r4": c.r4,
        "c_h": hc, "c_z1": zc1, "c_z2": zc2,
        "corners": np.array(CORNERS, np.int32), "rs": np.int32(RS),
    }


def run_build(lib_path, inp_path, out_path):
    """in a fresh process: drive one reference build through its C ABI"""
    d = dict(np.load(inp_path))
    lib = C.CDLL(str(lib_path))
    PF = C.POINTER(C.c_float)
    I = lambda v: C.byref(C.c_int(int(v)))
    F = lambda a: np.ascontiguousarray(a, np.float32).ctypes.data_as(PF)
    keep = []

    def full(v, nx):
        a = np.ascontiguousarray(np.repeat(np.asarray(v, np.float32)[:, None], nx, axis=1))
        keep.append(a)
        return a

    lib.gcomcot_init_gpu_()

    def init_layer(lid, parent, level, rel_time, nx, ny, h, z, r):
        corners = np.array(CORNERS if parent != -1 else [1, nx, 1, ny], np.int32)
        keep.append(corners)
        for a in r.values():
            keep.append(a)
        keep.extend([h, z])
        lib.gcomcot_init_layer_(I(lid), I(parent), I(level), I(RS if parent != -1 else 1), I(rel_time),
                                corners.ctypes.data_as(C.POINTER(C.c_int)), C.byref(C.c_float(0.0)),
                                C.byref(C.c_float(0.0)), F(r["r1"]), F(r["r2"]), F(r["r3"]), F(r["r4"]),
                                F(r["r5"]), F(r["r6"]), F(r["r11"]), F(h), F(z), I(nx), I(ny))

    pr = {"r1": full(d["p_r1"], PNX), "r11": full(d["p_r11"], PNX), "r3": full(d["p_r3"], PNX),
          "r5": full(d["p_r5"], PNX), "r2": np.ascontiguousarray(d["p_r2"]), "r4": np.ascontiguousarray(d["p_r4"]),
          "r6": np.ascontiguousarray(d["p_r6"])}
    zeros_c = np.zeros((CNY, CNX), np.float32)
    cr = {k: zeros_c for k in ("r1", "r11", "r3", "r5", "r2", "r4")}
    cr["r6"] = np.zeros(CNY, np.float32)
    h_p = np.ascontiguousarray(d["p_h"], np.float32)
    zmax0 = np.ascontiguousarray(d["p_zmax"], np.float32)
    init_layer(1, -1, 1, 1, PNX, PNY, h_p, zmax0, pr)
    h_c = np.ascontiguousarray(d["c_h"], np.float32)
    init_layer(2, 1, 2, REL_TIME, CNX, CNY, h_c, np.ascontiguousarray(d["c_z1"], np.float32), cr)
    out = {}

    def get_z(lid, nx, ny):
        a = np.zeros((ny, nx), np.float32)
        lib.cuda_getz_(a.ctypes.data_as(PF), I(lid))
        return a

    def get_mn1(lid, nx, ny):
        m = np.zeros((ny, nx), np.float32)
        n = np.zeros((ny, nx), np.float32)
        lib.cuda_getmn1_(m.ctypes.data_as(PF), n.ctypes.data_as(PF), I(lid))
        return m, n

    # ---- mass + max recorder on layer 1 ----
    z1 = np.ascontiguousarray(d["p_z1"]); m1 = np.ascontiguousarray(d["p_m1"]); n1 = np.ascontiguousarray(d["p_n1"])
    lib.cuda_setz1_(z1.ctypes.data_as(PF), I(1))
    lib.cuda_setmn1_(m1.ctypes.data_as(PF), n1.ctypes.data_as(PF), I(1))
    lib.mass_launch_(None, None, None, I(1))
    out["mass_z2"] = get_z(1, PNX, PNY)
    lib.maxamp_launch_(I(1))
    zm = np.zeros((PNY, PNX), np.float32)
    lib.cuda_getzmax_(zm.ctypes.data_as(PF), I(1))
    out["maxamp"] = zm
    # ---- edge fluxes: parent Z2/M1/N1 and child H/Z1 as inputs ----
    z2 = np.ascontiguousarray(d["p_z2"])
    lib.cuda_setz_(z2.ctypes.data_as(PF), I(1))
    lib.cuda_setmn1_(m1.ctypes.data_as(PF), n1.ctypes.data_as(PF), I(1))
    cz1 = np.ascontiguousarray(d["c_z1"]); cz2 = np.ascontiguousarray(d["c_z2"])
    lib.cuda_setz1_(cz1.ctypes.data_as(PF), I(2))
    zc = np.zeros((CNY, CNX), np.float32)
    lib.cuda_setmn1_(zc.ctypes.data_as(PF), zc.ctypes.data_as(PF), I(2))
    # host comparison buffers the debug entry point reads (its prints are noise here)
    hm = np.zeros((CNY, CNX), np.float32); hn = np.zeros((CNY, CNX), np.float32)
    yf = np.zeros(2 * PNY, np.float32); xf = np.zeros(2 * PNX, np.float32)
    mO = np.zeros((PNY, PNX), np.float32)
    for t in (1, 2, 3):
        lib.edgeinterp_dbglaunch_(mO.ctypes.data_as(PF), mO.ctypes.data_as(PF), I(1), hm.ctypes.data_as(PF),
                                  hn.ctypes.data_as(PF), I(2), I(t), yf.ctypes.data_as(PF), xf.ctypes.data_as(PF))
        m, n = get_mn1(2, CNX, CNY)
        out[f"edge{t}_m"] = m
        out[f"edge{t}_n"] = n
    # ---- JNZ: child Z1, Z2, H -> parent Z2 over the window ----
    lib.cuda_setz_(cz2.ctypes.data_as(PF), I(2))
    lib.cuda_setz_(z2.ctypes.data_as(PF), I(1))
    pz = np.zeros((PNY, PNX), np.float32)
    lib.jnz_dbglaunch_(pz.ctypes.data_as(PF), I(1), I(2))
    out["jnz_z2"] = get_z(1, PNX, PNY)
    np.savez(out_path, **out)


def main():
    if len(sys.argv) == 4 and sys.argv[1] == "--child":
        run_build(sys.argv[2], sys.argv[3], sys.argv[3] + ".out.npz")
        return 0
    inp = make_inputs()
    tmp = pathlib.Path(os.environ.get("TMPDIR", "/tmp")) / "ref_goldens_inputs.npz"
    np.savez(tmp, **inp)
    result = dict(inp)
    for tag, name in (("fma", "libref_gpu.so"), ("nofma", "libref_gpu_nofma.so")):
        lib = HERE / "_ref" / name
        subprocess.run([sys.executable, __file__, "--child", str(lib), str(tmp)], check=True,
                       stdout=subprocess.DEVNULL)
        got = dict(np.load(str(tmp) + ".out.npz"))
        for k, v in got.items():
            result[f"{tag}_{k}"] = v
    result["meta"] = np.array(json.dumps({"rel_time": REL_TIME, "pnx": PNX, "pny": PNY, "cnx": CNX,
                                          "cny": CNY}))
    OUT.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(OUT, **result)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
