"""The CPU oracle against golden vectors produced by the reference's own CUDA
kernels (built from their sources, driven through the reference C ABI; see
oracle/make_ref_goldens.py).  Where the reference kernel evaluates the same
float expression in the same order (MASS_S, the max recorder), the -fmad=false
build must agree bit for bit and the reference's own build within its
comparator tolerance (debug_option.h:12, absolute 1e-4).  The edge and JNZ
kernels compute in a different order (double-precision edge arithmetic,
GPUall_grids.cu:254-260; tree reduction, :545-564), so they are compared at
a relative 1e-6."""
import ctypes as C
import json
import pathlib

import numpy as np
import pytest

GOLD = pathlib.Path(__file__).resolve().parent / "golden" / "ref_kernels.npz"

pytestmark = pytest.mark.skipif(not GOLD.exists(), reason="golden vectors not generated yet")


def _setup(oracle_mod, d):
    meta = json.loads(str(d["meta"]))
    PNX, PNY, CNX, CNY = meta["pnx"], meta["pny"], meta["cnx"], meta["cny"]
    lib = oracle_mod.load(np.float32)
    arr = (oracle_mod.OLayer * 2)()
    keep = []

    def A(x, dt=np.float32):
        a = np.ascontiguousarray(np.array(x, dtype=dt))
        keep.append(a)
        return a

    P, Cc = arr[0], arr[1]
    corners = list(d["corners"])
    P.id, P.parent, P.level, P.nx, P.ny = 1, -1, 1, PNX, PNY
    P.rel_size = P.rel_time = 1
    Cc.id, Cc.parent, Cc.level, Cc.nx, Cc.ny = 2, 1, 2, CNX, CNY
    Cc.rel_size, Cc.rel_time = int(d["rs"]), meta["rel_time"]
    for q in range(4):
        P.corners[q] = [1, PNX, 1, PNY][q]
        Cc.corners[q] = int(corners[q])
    f = {}
    f["p"] = dict(r1=A(d["p_r1"]), r11=A(d["p_r11"]), r6=A(d["p_r6"]), r3=A(d["p_r3"]), r5=A(d["p_r5"]),
                  r2=A(d["p_r2"]), r4=A(d["p_r4"]), h=A(d["p_h"]), hp=A(np.zeros((PNY, PNX))),
                  hq=A(np.zeros((PNY, PNX))), z1=A(d["p_z1"]), z2=A(np.zeros((PNY, PNX))), m1=A(d["p_m1"]),
                  m2=A(np.zeros((PNY, PNX))), n1=A(d["p_n1"]), n2=A(np.zeros((PNY, PNX))),
                  dz2=A(np.zeros((PNY, PNX))), xflux=A(np.zeros(2 * PNX)), yflux=A(np.zeros(2 * PNY)),
                  zmax=A(d["p_zmax"]))
    zc = np.zeros((CNY, CNX))
    f["c"] = dict(r1=A(np.zeros(CNY)), r11=A(np.zeros(CNY)), r6=A(np.zeros(CNY)), r3=A(np.zeros(CNY)),
                  r5=A(np.zeros(CNY)), r2=A(zc), r4=A(zc), h=A(d["c_h"]), hp=A(zc), hq=A(zc), z1=A(d["c_z1"]),
                  z2=A(d["c_z2"]), m1=A(zc), m2=A(zc), n1=A(zc), n2=A(zc), dz2=A(zc), xflux=A(np.zeros(2 * CNX)),
                  yflux=A(np.zeros(2 * CNY)), zmax=None)
    for o, key in ((P, "p"), (Cc, "c")):
        for nm, a in f[key].items():
            setattr(o, nm, a.ctypes.data if a is not None else None)
        o.arrival = None
    return lib, arr, f, meta


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(GOLD))


def test_mass_bitwise_against_reference_kernel(oracle_mod, gold):
    lib, arr, f, m = _setup(oracle_mod, gold)
    lib.ocl_mass(C.addressof(arr[0]))
    z2 = f["p"]["z2"]
    inner = (slice(1, m["pny"] - 1), slice(1, m["pnx"] - 1))
    assert np.array_equal(z2[inner].view(np.uint32), gold["nofma_mass_z2"][inner].view(np.uint32))
    assert np.abs(z2[inner] - gold["fma_mass_z2"][inner]).max() <= 1e-4
    # the max recorder: Zmax starts from the initial surface
    zmax = np.where(gold["p_zmax"] >= z2, gold["p_zmax"], z2)
    assert np.array_equal(zmax[inner], gold["nofma_maxamp"][inner])


@pytest.mark.parametrize("t", [1, 2, 3])
def test_edge_fluxes_against_reference_kernel(oracle_mod, gold, t):
    lib, arr, f, m = _setup(oracle_mod, gold)
    P, Cc = C.addressof(arr[0]), C.addressof(arr[1])
    f["p"]["z2"][...] = gold["p_z2"]
    # JNQ at T=1, then NEWQ at T=2 (forecast into the cache) and T=3 (cache blend)
    for tt in range(1, t + 1):
        if tt == 1:
            lib.ocl_jnq(P, Cc)
        else:
            lib.ocl_newq(P, Cc, tt)
    cm, cn = f["c"]["m1"], f["c"]["n1"]
    for build in ("nofma", "fma"):
        gm, gn = gold[f"{build}_edge{t}_m"], gold[f"{build}_edge{t}_n"]
        for got, want in ((cm[1:, 0], gm[1:, 0]), (cm[1:, -1], gm[1:, -1]), (cn[0, 1:], gn[0, 1:]),
                          (cn[-1, 1:], gn[-1, 1:])):
            scale = max(float(np.abs(want).max()), 1e-20)
            assert np.abs(got - want).max() <= 1e-6 * scale + 1e-12
            assert np.array_equal(got == 0, want == 0)     # the same wet/dry zeros


def test_jnz_against_reference_kernel(oracle_mod, gold):
    lib, arr, f, m = _setup(oracle_mod, gold)
    f["p"]["z2"][...] = gold["p_z2"]
    lib.ocl_jnz(C.addressof(arr[0]), C.addressof(arr[1]))
    is_, ie, js, je = [int(x) for x in gold["corners"]]
    win = (slice(js - 1, je), slice(is_ - 1, ie))
    for build in ("nofma", "fma"):
        want = gold[f"{build}_jnz_z2"][win]
        got = f["p"]["z2"][win]
        scale = float(np.abs(want).max())
        assert np.abs(got - want).max() <= 1e-6 * scale
        assert np.array_equal(got == 0, want == 0)
