"""gcomcot_fused_step_noalloc: the step for callers that cannot allocate
device memory (they own every device array and pass it in; the library keeps
its work list in a fixed array of its own).  Checked against the batched
engine -- the existing entry point over the same fused kernel -- on two calls
in a row.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from comcot_b200 import _lib, synth
from comcot_b200.engine import Engine

pytestmark = pytest.mark.gpu

TOL = 1e-4  # the parity tolerance used throughout the GPU tests


class StepIO(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("pitch", C.c_int),
                ("z1", C.c_void_p), ("m1", C.c_void_p), ("n1", C.c_void_p),
                ("z2", C.c_void_p), ("m2", C.c_void_p), ("n2", C.c_void_p),
                ("h", C.c_void_p), ("rows", C.c_void_p), ("zmax", C.c_void_p)]


def _case(nx, ny, seed):
    return synth.single_layer_case("na", nx, ny, 2.0, 2.0, 2, seed=seed, n_seamounts=3,
                                   shelf_cols=max(2, nx // 10), land_cols=max(1, nx // 30), source="dipole",
                                   amp=2.0)


def test_noalloc_step_matches_engine_on_two_calls():
    import torch

    lib = _lib.load()
    cases = [_case(97, 81, 61), _case(150, 70, 62), _case(61, 45, 63)]
    dev = torch.device("cuda", 0)

    def pitched(a, pitch):
        t = torch.zeros((a.shape[0], pitch), dtype=torch.float32, device=dev)
        t[:, :a.shape[1]] = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(dev)
        return t

    bufs = []
    for c in cases:
        L = c.root
        pitch = (L.nx + 31) // 32 * 32
        rec = np.zeros((L.ny, 8), np.float32)
        rec[:, :7] = L.coefs.rows().T
        zero = lambda: torch.zeros((L.ny, pitch), dtype=torch.float32, device=dev)
        bufs.append({"nx": L.nx, "ny": L.ny, "pitch": pitch,
                     "z": [pitched(L.Z0, pitch), zero()], "m": [zero(), zero()], "n": [zero(), zero()],
                     "h": pitched(L.H, pitch), "rows": torch.from_numpy(rec).to(dev),
                     "zmax": pitched(L.Z0, pitch)})
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev).cuda_stream
    for k in range(2):                      # two calls in a row: level 1 -> 2, then back
        src, dst = k % 2, 1 - k % 2
        arr = (StepIO * len(bufs))()
        for g, b in enumerate(bufs):
            q = arr[g]
            q.nx, q.ny, q.pitch = b["nx"], b["ny"], b["pitch"]
            q.z1, q.m1, q.n1 = b["z"][src].data_ptr(), b["m"][src].data_ptr(), b["n"][src].data_ptr()
            q.z2, q.m2, q.n2 = b["z"][dst].data_ptr(), b["m"][dst].data_ptr(), b["n"][dst].data_ptr()
            q.h, q.rows, q.zmax = b["h"].data_ptr(), b["rows"].data_ptr(), b["zmax"].data_ptr()
        rc = lib.gcomcot_fused_step_noalloc(len(bufs), C.cast(arr, C.c_void_p), C.c_void_p(stream))
        assert rc == 0
    torch.cuda.synchronize()

    # the existing entry point: the same members in the batched engine, two steps
    with Engine(budget=1 << 30) as eng:
        ids = [eng.add(c, nsteps=2, gauges=[], arrival_thr=-1.0) for c in cases]
        eng.step(3)
        eng.sync()
        for b, mid in zip(bufs, ids):
            ref = eng.read(mid)
            nx = b["nx"]
            got = {"z": b["z"][0][:, :nx].cpu().numpy(), "m": b["m"][0][:, :nx].cpu().numpy(),
                   "n": b["n"][0][:, :nx].cpu().numpy(), "zmax": b["zmax"][:, :nx].cpu().numpy()}
            for key in ("z", "m", "n", "zmax"):
                want = ref[key]
                scale = max(float(np.abs(want).max()), 1e-30)
                assert float(np.abs(got[key].astype(np.float64) - want).max()) <= TOL * scale, key
                # the same kernel and arithmetic: identical bits as well
                assert np.array_equal(got[key].view(np.uint32), want.view(np.uint32)), key

    # sizes beyond the fixed array are refused, before any device work
    many = (StepIO * 65)()
    assert lib.gcomcot_fused_step_noalloc(65, C.cast(many, C.c_void_p), C.c_void_p(stream)) == -1
