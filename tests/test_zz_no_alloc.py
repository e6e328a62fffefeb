"""gcomcot_fused_step_noalloc: the step for callers that cannot allocate
device memory (they own every device array and pass it in; the library keeps
its work list in a fixed array of its own).  Checked against the batched
engine -- the existing entry point over the same fused kernel -- and against
the FP32 oracle on two calls in a row; on a grid whose work list only fits the
fixed array once the tile height is raised; and refused, before any device
work, where it fits at no height.  Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from comcot_b200 import _lib, synth
from comcot_b200.engine import Engine

pytestmark = pytest.mark.gpu

TOL = 1e-4  # the parity tolerance used throughout the GPU tests
MAX_TILES = 24576  # the fixed work list's capacity, in 128-column tiles


class StepIO(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("pitch", C.c_int),
                ("z1", C.c_void_p), ("m1", C.c_void_p), ("n1", C.c_void_p),
                ("z2", C.c_void_p), ("m2", C.c_void_p), ("n2", C.c_void_p),
                ("h", C.c_void_p), ("rows", C.c_void_p), ("zmax", C.c_void_p)]


def _case(nx, ny, seed, **kw):
    return synth.single_layer_case("na", nx, ny, kw.pop("dx", 2.0), kw.pop("dt", 2.0), 2, seed=seed,
                                   n_seamounts=3, shelf_cols=max(2, nx // 10), land_cols=max(1, nx // 30),
                                   source="dipole", amp=2.0, **kw)


def _buffers(cases, dev):
    """each grid's arrays as the caller owns them: pitched device tensors"""
    import torch

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
    return bufs


def _two_calls(lib, bufs, stream):
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


def _results(b):
    nx = b["nx"]
    return {"z": b["z"][0][:, :nx].cpu().numpy(), "m": b["m"][0][:, :nx].cpu().numpy(),
            "n": b["n"][0][:, :nx].cpu().numpy(), "zmax": b["zmax"][:, :nx].cpu().numpy()}


def _check(got, want, what):
    scale = max(float(np.abs(want).max()), 1e-30)
    assert float(np.abs(got.astype(np.float64) - want).max()) <= TOL * scale, what
    # the same kernel and arithmetic: identical bits as well
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), what


def _against_engine(cases, bufs):
    with Engine(budget=16 << 30) as eng:
        ids = [eng.add(c, nsteps=2, gauges=[], arrival_thr=-1.0) for c in cases]
        eng.step(3)
        eng.sync()
        for b, mid in zip(bufs, ids):
            ref = eng.read(mid, fields=("z", "m", "n", "zmax"))
            got = _results(b)
            for key in ("z", "m", "n", "zmax"):
                _check(got[key], ref[key], "engine " + key)


def test_noalloc_step_matches_engine_and_oracle_on_two_calls(oracle_mod):
    import torch

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    cases = [_case(97, 81, 61), _case(150, 70, 62), _case(61, 45, 63)]
    bufs = _buffers(cases, dev)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev).cuda_stream
    _two_calls(lib, bufs, stream)
    torch.cuda.synchronize()
    assert lib.gcomcot_sync() == 0  # no bounded wait gave up
    _against_engine(cases, bufs)
    for c, b in zip(cases, bufs):
        o = oracle_mod.OracleRun(c)
        o.run(2, arrival=False)
        ref = o.layer(0)
        got = _results(b)
        for key in ("z", "m", "n", "zmax"):
            _check(got[key], ref[key], "oracle " + key)

    # sizes beyond the fixed array are refused, before any device work
    many = (StepIO * 65)()
    assert lib.gcomcot_fused_step_noalloc(65, C.cast(many, C.c_void_p), C.c_void_p(stream)) == -1


def test_noalloc_raises_tile_height_until_the_work_list_fits():
    """4096 x 16384 cells: 32 x 1024 = 32768 tiles at the 16-row height, more
    than the fixed list holds, so the call takes taller tiles"""
    import torch

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    nx, ny = 4096, 16384
    assert (nx // 128) * (ny // 16) > MAX_TILES
    cases = [_case(nx, ny, 64, dx=0.25, dt=0.5, lat0=-34.0)]
    bufs = _buffers(cases, dev)
    torch.cuda.synchronize()
    _two_calls(lib, bufs, torch.cuda.current_stream(dev).cuda_stream)
    torch.cuda.synchronize()
    assert lib.gcomcot_sync() == 0
    _against_engine(cases, bufs)
    del bufs
    torch.cuda.empty_cache()


def test_noalloc_refuses_a_grid_that_fits_at_no_height():
    """24577 tiles across: more than the list holds even at one tile per column"""
    import torch

    lib = _lib.load()
    dev = torch.device("cuda", 0)
    nx, ny = MAX_TILES * 128 + 1, 3
    pitch = (nx + 31) // 32 * 32
    f = [torch.zeros((ny, pitch), dtype=torch.float32, device=dev) for _ in range(8)]
    rows = torch.zeros((ny, 8), dtype=torch.float32, device=dev)
    q = (StepIO * 1)()
    q[0].nx, q[0].ny, q[0].pitch = nx, ny, pitch
    q[0].z1, q[0].m1, q[0].n1, q[0].z2, q[0].m2, q[0].n2, q[0].h, q[0].zmax = (t.data_ptr() for t in f)
    q[0].rows = rows.data_ptr()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev).cuda_stream
    assert lib.gcomcot_fused_step_noalloc(1, C.cast(q, C.c_void_p), C.c_void_p(stream)) == -1
    torch.cuda.synchronize()
    assert float(f[3].abs().max()) == 0.0  # nothing was written
