"""On-device Okada source generation (gc_okada_apply) against the oracle's
restatement of deform.f90, and an engine member created from fault
parameters against the oracle run from the same initial state."""
import ctypes as C

import numpy as np
import pytest

from comcot_b200 import _lib, synth
from comcot_b200.engine import Engine

pytestmark = pytest.mark.gpu

FAULTS = [dict(hh=5000.0, l=60000.0, w=30000.0, d=3.0, th=30.0, dl=20.0, rd=90.0, sw=0),
          dict(hh=8000.0, l=40000.0, w=20000.0, d=2.0, th=210.0, dl=35.0, rd=60.0, sw=9)]


def _case():
    c = synth.single_layer_case("ok", 97, 81, 2.0, 2.0, 40, seed=9, n_seamounts=3, shelf_cols=8, land_cols=3,
                                ngauges=3)
    L = c.root
    faults = [dict(FAULTS[0], x0=float(L.x[40]), y0=float(L.y[38])),
              dict(FAULTS[1], x0=float(L.x[55]), y0=float(L.y[45]))]
    return c, faults


def _gpu_apply(faults, laycord, nx, ny, x, y, dx, dy, z0, h0):
    import torch

    dev = torch.device("cuda", 0)
    pitch = (nx + 31) // 32 * 32
    z = torch.zeros((ny, pitch), dtype=torch.float32, device=dev)
    h = torch.zeros((ny, pitch), dtype=torch.float32, device=dev)
    z[:, :nx] = torch.from_numpy(np.ascontiguousarray(z0, np.float32)).to(dev)
    h[:, :nx] = torch.from_numpy(np.ascontiguousarray(h0, np.float32)).to(dev)
    xd = torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(dev)
    yd = torch.from_numpy(np.ascontiguousarray(y, np.float32)).to(dev)
    arr = _lib.faults_array(faults)
    torch.cuda.synchronize()
    rc = _lib.load().gc_okada_apply(C.cast(arr, C.c_void_p), len(faults), laycord, nx, ny, pitch, xd.data_ptr(),
                                    yd.data_ptr(), dx, dy, z.data_ptr(), h.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    return z[:, :nx].cpu().numpy(), h[:, :nx].cpu().numpy()


@pytest.mark.parametrize("laycord", [0, 1])
def test_okada_matches_double_restatement(oracle_mod, laycord):
    c, faults = _case()
    L = c.root
    x = L.x.astype(np.float32).astype(np.float64)       # the device reads float axes
    y = L.y.astype(np.float32).astype(np.float64)
    if laycord == 1:
        # a Cartesian cell sits at DX*(I-1) - XL, XL the origin's offset from
        # the epicentre (deform.f90:150-154): an origin east and north of the
        # epicentre puts the fault inside the layer
        faults = [dict(f, xo=f["x0"] + 0.8, yo=f["y0"] + 0.6) for f in faults]
    dx = dy = 3000.0
    z0 = np.zeros_like(L.H)
    zg, hg = _gpu_apply(faults, laycord, L.nx, L.ny, x, y, dx, dy, z0, L.H)
    z64, h64 = oracle_mod.okada_apply(faults, laycord, L.nx, L.ny, x, y, dx, dy, z0, L.H, dtype=np.float64)
    scale = float(np.abs(z64).max())
    assert scale > 1e-3
    # double evaluation on both sides, the device result rounded to float per fault
    assert float(np.abs(zg - z64).max()) <= 1e-6 * scale + 1e-6
    assert np.all(np.abs(hg - h64) <= 2.0 ** -21 * np.abs(h64) + 1e-6)
    # the reference's float evaluation: its terms are O(1) before they cancel,
    # so it carries ~1e-6 m of rounding, and it jumps atan branches on the
    # lines through the fault ends; elsewhere it agrees
    z32, _ = oracle_mod.okada_apply(faults, laycord, L.nx, L.ny, x, y, dx, dy, z0, L.H, dtype=np.float32)
    assert (np.abs(zg - z32) > 1e-4 * scale + 2e-5).mean() < 0.005


def test_engine_member_from_faults_matches_oracle(oracle_mod):
    c, faults = _case()
    L = c.root
    zg, hg = _gpu_apply(faults, 0, L.nx, L.ny, L.x, L.y, 0.0, 0.0, np.zeros_like(L.H), L.H)
    with Engine(budget=1 << 30) as eng:
        mid = eng.add_faults(c, faults)
        eng.step(c.nsteps + 1)
        eng.sync()
        got = eng.read(mid)
    # the oracle from the same initial state: surface = deformation, depth =
    # H - deformation, and PARA / PQ_DEPTH on that depth (the reference runs
    # them after UPDATE_BATH, comcot.f90:199-215,683)
    Lo = synth.spherical_layer(1, L.x, L.y, hg, zg, L.dt, L.dx)
    case_o = synth.Case("okref", [Lo], c.nsteps, gauges=c.gauges, arrival_thr=c.arrival_thr)
    o = oracle_mod.OracleRun(case_o)
    ts = o.run(c.nsteps)
    ref = o.layer(0)
    for k in ("z", "m", "n", "zmax"):
        assert np.array_equal(got[k].view(np.uint32), ref[k].view(np.uint32)), k
    assert np.array_equal(got["arrival"], ref["arrival"])
    assert np.array_equal(got["ts"].view(np.uint32), ts.view(np.uint32))


def test_served_fault_request_equals_engine_member():
    from comcot_b200.serving import ForecastServer, Request

    c, faults = _case()
    with ForecastServer(budget_bytes=1 << 30, chunk=8) as srv:
        reqs = [Request(0, 0.0, c, faults=faults), Request(1, 0.0, c)]
        srv.serve(reqs, speed=float("inf"))
    assert [r.status for r in reqs] == ["done", "done"]
    with Engine(budget=1 << 30) as eng:
        mid = eng.add_faults(c, faults)
        eng.step(c.nsteps + 1)
        eng.sync()
        alone = eng.read(mid)
    for k in ("zmax", "ts"):
        assert np.array_equal(reqs[0].result[k].view(np.uint32), alone[k].view(np.uint32)), k
